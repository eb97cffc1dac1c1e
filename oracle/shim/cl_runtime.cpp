// Registry and thread settings of the fake OpenCL runtime (oracle only).
//
// TEST INFRASTRUCTURE ONLY.
#include <CL/cl.hpp>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>

#include "clc_shim.h"

namespace clshim {

thread_local WorkItem g_wi;

namespace {
std::map<std::string, Launcher>& table() {
    static std::map<std::string, Launcher> t;
    return t;
}
std::string& next_program() {
    static std::string p;
    return p;
}
int g_threads = 1;
}  // namespace

void register_kernel(const std::string& program, const std::string& name, Launcher fn) {
    table()[program + "/" + name] = std::move(fn);
}

const Launcher& find_kernel(const std::string& program, const std::string& name) {
    auto it = table().find(program + "/" + name);
    if (it == table().end()) {
        std::fprintf(stderr, "oracle: kernel %s/%s not registered\n", program.c_str(), name.c_str());
        throw cl::Error(-46, "kernel not registered");
    }
    return it->second;
}

void set_next_program(const std::string& id) { next_program() = id; }
std::string current_next_program() { return next_program(); }

void set_num_threads(int n) { g_threads = n < 1 ? 1 : n; }
int num_threads() { return g_threads; }

}  // namespace clshim
