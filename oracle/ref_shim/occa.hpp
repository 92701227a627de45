// ORACLE test infrastructure: a minimal stand-in for the OCCA v0 API that
// the reference's deviceclass uses (device / memory / kernel / kernelInfo),
// implementing its Serial and OpenMP modes.  buildKernelFromSource turns the
// .okl file into C++ by the handful of token rewrites OKL v0 needs (the
// 4-clause outer/inner for-loops, `shared`, `barrier`, `occaUnroll`,
// `restrict`), prepends the kernelInfo defines and compiles it with g++ into
// a cached shared object that is dlopen'ed.
//
// Two environment hooks make the reference's own runs usable as test
// fixtures without changing its sources:
//   ESDG_REF_DUMP=<dir>   every memory.copyFrom(host) is written to
//                         <dir>/from_NNN.bin, and the last memory.copyTo(host)
//                         of each buffer to <dir>/to_MMM.bin (manifest.txt
//                         maps sequence numbers to buffers);
//   ESDG_REF_INJECT=<dir> a copyFrom(host) with sequence number NNN takes its
//                         bytes from <dir>/from_NNN.bin when that file exists
//                         (same size required), i.e. a chosen initial state
//                         and bathymetry replace the testcase's;
//   ESDG_REF_COUNT=1      at exit, the number of calls of every kernel is
//                         printed ("[occa shim] calls <kernel> <n>"), which
//                         gives the number of time steps a run took.
#pragma once

#include <cstddef>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace occa {

void printAvailableDevices();

class memory {
  public:
    struct Impl {
        void* ptr = nullptr;
        size_t bytes = 0;
        int id = -1;
    };
    Impl* p = nullptr;
    memory() {}
    explicit memory(Impl* i) : p(i) {}
    void copyFrom(const void* src);
    void copyFrom(const memory& m);
    void copyTo(void* dst) const;
    void free();
    size_t size() const { return p ? p->bytes : 0; }
    void* ptr() const { return p ? p->ptr : nullptr; }
    // src/deviceclass.cpp:1301 passes a memory object to C free()
    operator void*() const { return ptr(); }
};

class kernelInfo {
  public:
    std::vector<std::pair<std::string, std::string>> defines;
    std::vector<std::string> flags;
    void addDefine(const std::string& n, const std::string& v) { defines.emplace_back(n, v); }
    void addDefine(const std::string& n, const char* v) { defines.emplace_back(n, std::string(v)); }
    void addDefine(const std::string& n, int v) { defines.emplace_back(n, std::to_string(v)); }
    void addDefine(const std::string& n, long v) { defines.emplace_back(n, std::to_string(v)); }
    void addDefine(const std::string& n, double v);
    void addDefine(const std::string& n, float v) { addDefine(n, (double)v); }
    void addCompilerFlag(const std::string& f) { flags.push_back(f); }
};

namespace detail {
template <class T, class Enable = void>
struct arg {
    typedef T type;
    static T conv(const T& v) { return v; }
};
template <class T>
struct arg<T, typename std::enable_if<std::is_integral<T>::value>::type> {
    typedef int type;
    static int conv(T v) { return (int)v; }
};
template <class T>
struct arg<T, typename std::enable_if<std::is_floating_point<T>::value>::type> {
    typedef double type;
    static double conv(T v) { return (double)v; }
};
template <>
struct arg<memory, void> {
    typedef void* type;
    static void* conv(const memory& m) { return m.ptr(); }
};
}  // namespace detail

void note_kernel_call(const std::string& name);

class kernel {
  public:
    void* fn = nullptr;
    std::string name;
    template <class... A>
    void operator()(const A&... a) const {
        note_kernel_call(name);
        typedef void (*F)(typename detail::arg<A>::type...);
        reinterpret_cast<F>(fn)(detail::arg<A>::conv(a)...);
    }
};

class device {
  public:
    std::string mode = "Serial";
    size_t allocated = 0;
    void setup(const std::string& s);
    memory malloc(size_t bytes, const void* src = nullptr);
    void finish() {}
    size_t bytesAllocated() const { return allocated; }
    kernel buildKernelFromSource(const std::string& file, const std::string& name, const kernelInfo& info);
};

}  // namespace occa
