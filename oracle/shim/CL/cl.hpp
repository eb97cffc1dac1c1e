// Fake OpenCL C++ bindings for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY.  The reference's host classes (DominoTiler.cpp,
// LozengeTiler.cpp, RectTriangleTiler.cpp, TriangleDimerTiler.cpp,
// common.cpp, file_reader.cpp) include <CL/cl.hpp>; pointing the include path
// here lets those files compile unmodified and run their kernels on the host.
//
// Only the subset of the Khronos cl.hpp API that the reference touches is
// provided.  Buffers are host byte vectors; "enqueuing" a kernel runs it over
// its NDRange immediately (in-order queue semantics), serially or with OpenMP
// over work items.  The kernels the reference launches are data-race free per
// launch (each work item writes only its own site of arrays it does not read
// at other sites), so any work-item order gives the same result.
#ifndef ORACLE_FAKE_CL_HPP
#define ORACLE_FAKE_CL_HPP

#include <cstddef>
#include <cstring>
#include <exception>
#include <functional>
#include <iterator>
#include <memory>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

typedef int cl_int;
typedef unsigned int cl_uint;
typedef unsigned long cl_ulong;
typedef cl_ulong cl_mem_flags;
typedef cl_ulong cl_device_type;
typedef cl_uint cl_bool;

#define CL_SUCCESS 0
#define CL_BUILD_PROGRAM_FAILURE -11
#define CL_FALSE 0
#define CL_TRUE 1
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_DEVICE_TYPE_DEFAULT (1 << 0)
#define CL_DEVICE_TYPE_CPU (1 << 1)
#define CL_DEVICE_TYPE_GPU (1 << 2)
#define CL_CONTEXT_DEVICES 0x1081
#define CL_PLATFORM_NAME 0x0902
#define CL_PLATFORM_VENDOR 0x0903
#define CL_DEVICE_TYPE 0x1000
#define CL_DEVICE_MAX_COMPUTE_UNITS 0x1002
#define CL_DEVICE_MAX_CLOCK_FREQUENCY 0x100C
#define CL_DEVICE_MAX_MEM_ALLOC_SIZE 0x1010
#define CL_DEVICE_LOCAL_MEM_SIZE 0x1023
#define CL_DEVICE_AVAILABLE 0x1027
#define CL_DEVICE_NAME 0x102B
#define CL_DEVICE_VENDOR 0x102C
#define CL_PROGRAM_BUILD_LOG 0x1183

namespace clshim {

// One kernel argument as the host passed it: a buffer's storage or a scalar.
struct Arg {
    void* ptr;
    long long ival;
};

// Runs a registered kernel over a global NDRange of `dims` dimensions.
typedef std::function<void(const std::vector<Arg>&, const size_t* gsize, int dims)> Launcher;

void register_kernel(const std::string& program, const std::string& name, Launcher fn);
const Launcher& find_kernel(const std::string& program, const std::string& name);

// The next cl::Program constructed binds to this kernel set ("domino",
// "domino_cftp", "lozenge", "qlozenge", "recttri", "tridimer").
void set_next_program(const std::string& id);
std::string current_next_program();

// Host threads used to run one NDRange (1 = serial, work-item order).
void set_num_threads(int n);
int num_threads();

}  // namespace clshim

namespace cl {

class Error : public std::exception {
    cl_int err_;
    const char* what_;

public:
    explicit Error(cl_int e, const char* w = "cl::Error") : err_(e), what_(w) {}
    cl_int err() const { return err_; }
    const char* what() const noexcept override { return what_; }
};

class Device {
public:
    template <cl_int Name>
    std::string getInfo() const { return "oracle-host-cpu"; }
    cl_int getInfo(cl_int, std::string* s) const {
        *s = "oracle-host-cpu";
        return CL_SUCCESS;
    }
};

class Platform {
public:
    static cl_int get(std::vector<Platform>* p) {
        p->assign(1, Platform());
        return CL_SUCCESS;
    }
    template <cl_int Name>
    std::string getInfo() const { return "oracle"; }
    cl_int getDevices(cl_device_type, std::vector<Device>* d) const {
        d->assign(1, Device());
        return CL_SUCCESS;
    }
};

class Context {
public:
    Context() {}
    explicit Context(cl_device_type) {}
    cl_int getInfo(cl_int, std::vector<Device>* d) const {
        d->assign(1, Device());
        return CL_SUCCESS;
    }
};

class Buffer {
    std::shared_ptr<std::vector<unsigned char> > mem_;

public:
    Buffer() {}
    Buffer(const Context&, cl_mem_flags, size_t size, void* host = nullptr)
        : mem_(std::make_shared<std::vector<unsigned char> >(size)) {
        if (host && size) std::memcpy(mem_->data(), host, size);
    }
    template <class It>
    Buffer(const Context&, It first, It last, bool /*readOnly*/, bool /*useHostPtr*/ = false) {
        typedef typename std::iterator_traits<It>::value_type T;
        const size_t n = static_cast<size_t>(std::distance(first, last));
        mem_ = std::make_shared<std::vector<unsigned char> >(n * sizeof(T));
        unsigned char* dst = mem_->data();
        for (It it = first; it != last; ++it, dst += sizeof(T)) {
            T v = *it;
            std::memcpy(dst, &v, sizeof(T));
        }
    }
    void* data() const { return mem_ ? mem_->data() : nullptr; }
    size_t size() const { return mem_ ? mem_->size() : 0; }
};

class CommandQueue {
public:
    CommandQueue() {}
    explicit CommandQueue(const Context&) {}
    cl_int enqueueWriteBuffer(const Buffer& b, cl_bool, size_t offset, size_t size, const void* ptr) const {
        if (offset + size > b.size()) throw Error(-30, "enqueueWriteBuffer out of range");
        std::memcpy(static_cast<unsigned char*>(b.data()) + offset, ptr, size);
        return CL_SUCCESS;
    }
    cl_int finish() const { return CL_SUCCESS; }
};

template <class It>
inline cl_int copy(const CommandQueue&, const Buffer& b, It first, It last) {
    typedef typename std::iterator_traits<It>::value_type T;
    const size_t n = static_cast<size_t>(std::distance(first, last));
    if (n * sizeof(T) > b.size()) throw Error(-30, "cl::copy out of range");
    const unsigned char* src = static_cast<const unsigned char*>(b.data());
    for (It it = first; it != last; ++it, src += sizeof(T)) {
        T v;
        std::memcpy(&v, src, sizeof(T));
        *it = v;
    }
    return CL_SUCCESS;
}

class NDRange {
    size_t sz_[3];
    int dims_;

public:
    NDRange() : sz_{0, 1, 1}, dims_(0) {}
    explicit NDRange(size_t a) : sz_{a, 1, 1}, dims_(1) {}
    NDRange(size_t a, size_t b) : sz_{a, b, 1}, dims_(2) {}
    NDRange(size_t a, size_t b, size_t c) : sz_{a, b, c}, dims_(3) {}
    const size_t* sizes() const { return sz_; }
    int dims() const { return dims_; }
};

class EnqueueArgs {
    NDRange global_;

public:
    EnqueueArgs(const CommandQueue&, NDRange global) : global_(global) {}
    EnqueueArgs(const CommandQueue&, NDRange global, NDRange) : global_(global) {}
    const NDRange& global() const { return global_; }
};

class Program {
    std::string id_;

public:
    typedef std::vector<std::pair<const char*, size_t> > Sources;
    Program() {}
    Program(const Context&, const Sources&, cl_int* err = nullptr) : id_(clshim::current_next_program()) {
        if (err) *err = CL_SUCCESS;
    }
    cl_int build(const std::vector<Device>&, const char* = nullptr) const { return CL_SUCCESS; }
    template <cl_int Name>
    std::string getBuildInfo(const Device&) const { return std::string(); }
    const std::string& id() const { return id_; }
};

namespace detail {
inline void push_arg(std::vector<clshim::Arg>& v, const Buffer& b) { v.push_back(clshim::Arg{b.data(), 0}); }
template <class T>
inline typename std::enable_if<std::is_arithmetic<T>::value>::type push_arg(std::vector<clshim::Arg>& v, T x) {
    v.push_back(clshim::Arg{nullptr, static_cast<long long>(x)});
}
}  // namespace detail

template <class... Ts>
class make_kernel {
    clshim::Launcher fn_;

public:
    make_kernel(const Program& p, const char* name) : fn_(clshim::find_kernel(p.id(), name)) {}
    void operator()(const EnqueueArgs& ea, Ts... args) const {
        std::vector<clshim::Arg> a;
        a.reserve(sizeof...(Ts));
        int unused[] = {0, (detail::push_arg(a, args), 0)...};
        (void)unused;
        fn_(a, ea.global().sizes(), ea.global().dims());
    }
};

}  // namespace cl

#endif  // ORACLE_FAKE_CL_HPP
