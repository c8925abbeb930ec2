// plugin.cu -- runtime network plug-ins compiled with NVRTC.
//
// Replaces the reference's build-time Precompiler (python/ode_systems/
// ode_base.py:16-123), which splices a network's RHS and Jacobian bodies into
// the solver sources and rebuilds the libraries.  Here the caller hands the
// same host plug-in source (the contract of cuda/include/ode_gold.h:1-12:
// calculate_dydt and calculate_jacobian over float arrays) to
// wind_plugin_create; it is compiled at run time for sm_100a with NVRTC:
//  * `float` is defined as `double` around the plug-in (the reference's
//    oracle build uses -Dfloat=double), so the network runs in FP64;
//  * -default-device makes its plain C functions device functions, and
//    --fmad=false keeps every product rounded before its add (bit-exact
//    with the reference's x86-64 CPU build);
//  * the plug-in is linked, in the same NVRTC program, to the team kernel of
//    plugin_kernel.cuh (whose sources are embedded in this library at build
//    time), one instantiation per (method, controller);
//  * the cubin is loaded per device with cudaLibraryLoadData and launched
//    through the kernel handles.
// NVRTC is opened with dlopen when the first plug-in is created: libwind
// does not depend on it otherwise.
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "api_internal.h"
#include "embedded_sources.h"
#include "plugin_kernel.cuh"

namespace wind {

// ---- NVRTC, opened at run time -------------------------------------------
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
    bool ok = false;
    std::string why;
    nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*,
                            const char* const*);
    nvrtcResult_t (*destroy)(nvrtcProgram_t*);
    nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*);
    nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*);
    nvrtcResult_t (*log)(nvrtcProgram_t, char*);
    nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*);
    nvrtcResult_t (*cubin)(nvrtcProgram_t, char*);
    nvrtcResult_t (*add_name)(nvrtcProgram_t, const char*);
    nvrtcResult_t (*lowered)(nvrtcProgram_t, const char*, const char**);
};

static Nvrtc& nvrtc() {
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnvrtc.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            n.why = "NVRTC (libnvrtc.so.12) not found";
            return;
        }
        bool all = true;
        auto sym = [&](const char* name) {
            void* p = dlsym(h, name);
            if (!p) all = false;
            return p;
        };
        n.create = (decltype(n.create))sym("nvrtcCreateProgram");
        n.destroy = (decltype(n.destroy))sym("nvrtcDestroyProgram");
        n.compile = (decltype(n.compile))sym("nvrtcCompileProgram");
        n.log_size = (decltype(n.log_size))sym("nvrtcGetProgramLogSize");
        n.log = (decltype(n.log))sym("nvrtcGetProgramLog");
        n.cubin_size = (decltype(n.cubin_size))sym("nvrtcGetCUBINSize");
        n.cubin = (decltype(n.cubin))sym("nvrtcGetCUBIN");
        n.add_name = (decltype(n.add_name))sym("nvrtcAddNameExpression");
        n.lowered = (decltype(n.lowered))sym("nvrtcGetLoweredName");
        n.ok = all;
        if (!all) n.why = "NVRTC library lacks an entry point";
    });
    return n;
}

// kernel instantiations, by (method, controller)
static const int kVariants[4][2] = {{WIND_METHOD_SIE, WIND_CTRL_DEVICE},
                                     {WIND_METHOD_SIE, WIND_CTRL_GOLD},
                                     {WIND_METHOD_RK2, WIND_CTRL_DEVICE},
                                     {WIND_METHOD_RK2, WIND_CTRL_GOLD}};

static std::string variant_name(int v) {
    char b[96];
    std::snprintf(b, sizeof b, "wind::k_plugin<wind::NetUser, %d, %d>", kVariants[v][0], kVariants[v][1]);
    return b;
}

}  // namespace wind

struct wind_plugin {
    int n_eq = 0, n_const = 0;
    std::vector<char> cubin;
    std::string lowered[4];
    std::mutex mu;
    struct Loaded {
        int device;
        cudaLibrary_t lib;
        cudaKernel_t k[4];
        int blocks_per_sm[4];
    };
    std::vector<Loaded> loaded;
};

using namespace wind;

static void put_log(char* log, int64_t log_size, const std::string& text) {
    if (!log || log_size <= 0) return;
    const size_t n = std::min<size_t>((size_t)log_size - 1, text.size());
    std::memcpy(log, text.data(), n);
    log[n] = '\0';
}

// Split `options` (whitespace-separated) into separate NVRTC options.
static std::vector<std::string> split_options(const char* options) {
    std::vector<std::string> out;
    if (!options) return out;
    std::string cur;
    for (const char* c = options; *c; c++) {
        if (*c == ' ' || *c == '\t' || *c == '\n') {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += *c;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

static int plugin_team_count(int n, int n_const) {
    // teams per block: up to a warp's worth of lanes x 4, bounded by ~96 KB
    // of shared memory per block
    const int ts = plugin_team(n);
    const size_t team_bytes = (size_t)(2 * n * n + 5 * n + (n_const > 0 ? n_const : 1)) * 8;
    int teams = PLUGIN_THREADS / ts;
    while (teams > 1 && (size_t)teams * team_bytes > 96 * 1024) teams /= 2;
    return teams;
}

extern "C" {

int wind_plugin_create(const char* source, int32_t n_eq, int32_t n_const, const char* options,
                       wind_plugin** out, char* log, int64_t log_size) {
    if (out) *out = nullptr;
    if (!source || !out || n_eq < 1 || n_const < 0) return WIND_ERR_ARGUMENT;
    if (n_eq > PLUGIN_MAX_EQ) return WIND_ERR_UNSUPPORTED;
    Nvrtc& nv = nvrtc();
    if (!nv.ok) {
        put_log(log, log_size, nv.why);
        return WIND_ERR_UNSUPPORTED;
    }
    // the program: the plug-in in FP64, then the kernel and the functor
    // that adapts the plug-in's contract to it
    std::string prog;
    prog += "#define float double\n#include \"ode_gold.h\"\n#line 1 \"plugin\"\n";
    prog += source;
    prog += "\n#undef float\n#include \"plugin_kernel.cuh\"\n";
    prog += "namespace wind {\nstruct NetUser {\n";
    prog += "    static constexpr int N = " + std::to_string(n_eq) + ";\n";
    prog += "    static constexpr int NC = " + std::to_string(n_const) + ";\n";
    prog += "    __device__ static void rhs(double t, const double* c, const double* y, double* f) {\n"
            "        calculate_dydt(t, const_cast<double*>(y), const_cast<double*>(c), f, N);\n    }\n"
            "    __device__ static void jac(const double* c, const double* y, double* J) {\n"
            "        calculate_jacobian(const_cast<double*>(y), const_cast<double*>(c), J);\n    }\n"
            "};\n}\n";
    // the plug-in's header (cuda/include/ode_gold.h:1-12 with NUM_CONST set)
    std::string ode_gold =
        "void calculate_dydt(float, float*, float*, float*, int);\n"
        "void calculate_jacobian(float*, float*, float*);\n"
        "#define NUM_CONST " + std::to_string(n_const) + "\n";
    std::vector<const char*> hdr_src, hdr_name;
    hdr_name.push_back("ode_gold.h");
    hdr_src.push_back(ode_gold.c_str());
    for (const char* libc : {"math.h", "stdio.h", "stdlib.h", "string.h"}) {
        hdr_name.push_back(libc);
        hdr_src.push_back("\n");
    }
    for (int i = 0; i < kEmbeddedCount; i++) {
        hdr_name.push_back(kEmbedded[i].name);
        hdr_src.push_back(kEmbedded[i].text);
    }
    nvrtcProgram_t p = nullptr;
    if (nv.create(&p, prog.c_str(), "wind_plugin.cu", (int)hdr_src.size(), hdr_src.data(),
                  hdr_name.data()) != 0) {
        put_log(log, log_size, "nvrtcCreateProgram failed");
        return WIND_ERR_UNSUPPORTED;
    }
    std::string names[4];
    for (int v = 0; v < 4; v++) {
        names[v] = variant_name(v);
        nv.add_name(p, names[v].c_str());
    }
    std::vector<std::string> opts = {"-arch=sm_100a", "-default-device", "--fmad=false", "-std=c++17",
                                     "-DWIND_PLUGIN_RTC=1"};
    for (auto& s : split_options(options)) opts.push_back(s);
    std::vector<const char*> optp;
    for (auto& s : opts) optp.push_back(s.c_str());
    const int rc = nv.compile(p, (int)optp.size(), optp.data());
    size_t ls = 0;
    nv.log_size(p, &ls);
    std::string text(ls, '\0');
    if (ls) nv.log(p, &text[0]);
    put_log(log, log_size, text);
    if (rc != 0) {
        nv.destroy(&p);
        return WIND_ERR_ARGUMENT;  // the plug-in source did not compile
    }
    auto* pl = new wind_plugin;
    pl->n_eq = n_eq;
    pl->n_const = n_const;
    size_t cs = 0;
    nv.cubin_size(p, &cs);
    pl->cubin.resize(cs);
    nv.cubin(p, pl->cubin.data());
    for (int v = 0; v < 4; v++) {
        const char* low = nullptr;
        nv.lowered(p, names[v].c_str(), &low);
        pl->lowered[v] = low ? low : "";
    }
    nv.destroy(&p);
    *out = pl;
    return WIND_OK;
}

int wind_plugin_destroy(wind_plugin* pl) {
    if (!pl) return WIND_ERR_ARGUMENT;
    for (auto& l : pl->loaded) cudaLibraryUnload(l.lib);
    delete pl;
    return WIND_OK;
}

int wind_integrate_plugin(const wind_options* opt_in, wind_plugin* pl, double tnow, double tend,
                          int32_t n_integration_steps, const double* constants, double* y,
                          int64_t nsys, double atol, double rtol, int32_t* sys_status,
                          int64_t* sys_nsteps, int64_t* total_nsteps, int32_t memory,
                          void* stream_v) {
    wind_options o;
    if (opt_in) o = *opt_in; else wind_default_options(&o);
    (void)cudaGetLastError();
    if (!pl || check_options(o) != WIND_OK) return WIND_ERR_ARGUMENT;
    // the plug-in path is the reference algorithm: Gauss-Jordan in FP64
    if (o.solver != WIND_SOLVER_GJE_F64 && o.solver != WIND_SOLVER_AUTO) return WIND_ERR_UNSUPPORTED;
    if (nsys < 0 || n_integration_steps < 1) return WIND_ERR_ARGUMENT;
    if (memory != WIND_MEM_HOST && memory != WIND_MEM_DEVICE) return WIND_ERR_ARGUMENT;
    if (nsys > 0 && (!y || (pl->n_const > 0 && !constants))) return WIND_ERR_ARGUMENT;
    if (total_nsteps) *total_nsteps = 0;
    if (nsys == 0) return WIND_OK;
    cudaStream_t stream = (cudaStream_t)stream_v;
    const int v = o.method * 2 + o.controller;
    // the cubin loaded on the current device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return launch_status("plugin device");
    cudaKernel_t kern = nullptr;
    int nb = 1;
    const int teams = plugin_team_count(pl->n_eq, pl->n_const);
    const int block = teams * plugin_team(pl->n_eq);
    const size_t smem = (size_t)teams * (2 * pl->n_eq * pl->n_eq + 5 * pl->n_eq +
                                         (pl->n_const > 0 ? pl->n_const : 1)) * sizeof(double);
    {
        std::lock_guard<std::mutex> g(pl->mu);
        wind_plugin::Loaded* L = nullptr;
        for (auto& l : pl->loaded)
            if (l.device == dev) L = &l;
        if (!L) {
            wind_plugin::Loaded n{};
            n.device = dev;
            wind_status st = cuda_status(
                cudaLibraryLoadData(&n.lib, pl->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0),
                "plugin load");
            if (st != WIND_OK) return st;
            for (int i = 0; i < 4; i++) {
                st = cuda_status(cudaLibraryGetKernel(&n.k[i], n.lib, pl->lowered[i].c_str()), "plugin kernel");
                if (st != WIND_OK) {
                    cudaLibraryUnload(n.lib);
                    return st;
                }
                cudaFuncSetAttribute((const void*)n.k[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                int b = 1;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)n.k[i], block, smem) != cudaSuccess ||
                    b < 1)
                    b = 1;
                (void)cudaGetLastError();
                n.blocks_per_sm[i] = b;
            }
            pl->loaded.push_back(n);
            L = &pl->loaded.back();
        }
        kern = L->k[v];
        nb = L->blocks_per_sm[v];
    }
    wind_network net{};
    net.kind = 0;
    net.n_eq = pl->n_eq;
    net.n_const = pl->n_const;
    net.constants = constants;
    IntegrateCall call;
    wind_status st = call.prepare(o, net, tnow, tend, n_integration_steps, y, nsys, atol, rtol, sys_status,
                                  sys_nsteps, memory, stream);
    if (st == WIND_OK) {
        const int64_t resident = (int64_t)nb * device_sm_count();
        const int64_t need = (nsys + teams - 1) / teams;
        const int grid = (int)(need < resident ? need : resident);
        void* args[] = {&call.params};
        st = cuda_status(cudaLaunchKernel((const void*)kern, dim3(grid), dim3(block), args, smem, stream),
                         "k_plugin launch");
        g_launches++;
    }
    if (st == WIND_OK) st = call.finish(total_nsteps);
    call.release();
    return st;
}

}  // extern "C"
