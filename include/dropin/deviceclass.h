// deviceclass.h for building the reference's own main.cpp against the B200
// engine: put this directory first on the include path, compile main.cpp and
// src/*.cpp except src/deviceclass.cpp, link libesdg_b200.so.  Includes what
// the reference header included (main.cpp relies on it) and maps the class
// name onto the C++ facade of the C ABI.
#ifndef DEVICECLASS_H
#define DEVICECLASS_H
#include "Constants.hpp"
#include "MPI_Communication.h"
#include "MPI_setup.h"
#include "MeshPartitioning.h"
#include "plots.h"
#include "RungeKutta.h"
#include "SW2D.h"
#include "basis.h"
#include "../esdg_deviceclass.hpp"
typedef esdg_dropin::deviceclass deviceclass;
#endif
