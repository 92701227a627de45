// main.cpp of the reference includes occa.hpp but uses no OCCA symbol
// itself once deviceclass is provided by the B200 engine; nothing to declare.
#pragma once
