// noalloc.cu — an RQMC pass for callers that cannot allocate GPU memory.
//
// Some callers of this library may not call cudaMalloc: code embedded in a host process whose
// device memory is owned by another allocator (a framework's caching allocator, a plugin host
// with a fixed memory budget), and latency-critical request paths where a cudaMalloc or
// cudaFree would synchronise the whole device at an unpredictable moment.  mcq_qmc_pass_noalloc
// serves them: the same fused pass as mcq_qmc_pass_device, but every byte of scratch it needs
// (the direction words scrambled for the call's replicas and the per-item partial sums) lives in
// one file-scope __device__ array of fixed size that is part of the loaded library.
//
// Limits: at most kMaxDims Sobol dimensions (steps x factors), kMaxReplicas replicas and
// kMaxItems work items; one-factor or Heston models without parameter arrays (GBM, Heston,
// parametric Dupire), raw noise ordering.  The array costs kScratchBytes (about 2.7 MiB) on
// every GPU that loads the library, held until the process exits.
//
// Sharing: every call uses the same array and it keeps the last call's contents.  Nothing in
// it has to start at zero: each call rewrites the scrambled words of its replicas before the
// pass reads them, and the pass writes every item record before the final reduction reads it.
// Two calls whose work overlaps on the GPU (for example on two streams at once) race on the
// array and produce wrong sums; issue them on one stream or synchronise in between.
//
// Set-up: every call resolves the array's device address with cudaGetSymbolAddress for the
// current device (a host-side lookup, no allocation).  The first call on each device, and the
// first call in a new context of that device (after a cudaDeviceReset the library's module and
// this array are loaded afresh, empty), copies the JoeKuo direction table for the first kMaxDims
// dimensions into the array with a synchronous cudaMemcpy.  That first call should therefore
// come before any stream capture.
//
// Work split and kernels: those of mcq_qmc_pass_device for the same request (the plain raw
// pass, or the packed pass with its whole-tile items for paths of at most 16 normals), so both
// entry points give the same sums bit for bit.
#include <cuda.h>
#include <cuda_runtime.h>
#include <curand.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "dispatch.h"
#include "engine.h"
#include "support.h"

namespace mcq {

constexpr int kMaxDims = 512;
constexpr int kMaxReplicas = 32;
// the work split of kTargetItems yields at most kTargetItems + R items, so every pass the
// allocating entry point runs (with the same split, hence the same sums) fits
constexpr int kMaxItems = 38912;
static_assert(kMaxItems >= kTargetItems + kMaxReplicas, "partials sized for the engine's work split");
constexpr size_t kTableBytes = (size_t)kMaxDims * 32 * sizeof(uint32_t);              // 64 KiB
constexpr size_t kDirsBytes = (size_t)kMaxReplicas * 33 * kMaxDims * sizeof(uint32_t); // 2.06 MiB
constexpr size_t kPartialBytes = (size_t)kMaxItems * 2 * sizeof(double);              // 608 KiB
constexpr size_t kScratchBytes = kTableBytes + kDirsBytes + kPartialBytes;
static_assert(kTableBytes % 256 == 0 && kDirsBytes % 256 == 0, "256-byte aligned sections");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch[kMaxDevices] = {};      // device address the table was loaded at
unsigned long long g_ctx_id[kMaxDevices] = {};   // context it was loaded in (driver context id)
int g_sm_count[kMaxDevices] = {};

// The driver's id of the current context (unique for the life of the process: a context
// created after a cudaDeviceReset has a new id), through the runtime's driver entry points.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        MCQ_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q));
        MCQ_REQUIRE(f && q == cudaDriverEntryPointSuccess, MCQ_ERR_CUDA, "cuCtxGetCurrent not available");
        get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        MCQ_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q));
        MCQ_REQUIRE(f && q == cudaDriverEntryPointSuccess, MCQ_ERR_CUDA, "cuCtxGetId not available");
        get_id = reinterpret_cast<GetId>(f);
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    MCQ_REQUIRE(get_current(&c) == CUDA_SUCCESS && c != nullptr, MCQ_ERR_CUDA, "no current CUDA context");
    MCQ_REQUIRE(get_id(c, &id) == CUDA_SUCCESS, MCQ_ERR_CUDA, "cuCtxGetId failed");
    return id;
}

// Every call, with the device current: resolve the array's device address (the host-side name
// g_noalloc_scratch is only a stand-in and must never be passed to a kernel), and load the
// direction table when this device's array has not been loaded in this context at this address.
unsigned char* scratch_for_current_device(int* sm_count) {
    int dev = -1;
    MCQ_CUDA(cudaGetDevice(&dev));
    MCQ_REQUIRE(dev >= 0 && dev < kMaxDevices, MCQ_ERR_RANGE, "device index beyond the set-up table");
    void* ptr = nullptr;
    MCQ_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    MCQ_REQUIRE(ptr != nullptr, MCQ_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (g_scratch[dev] != ptr || g_ctx_id[dev] != ctx) {
        curandDirectionVectors32_t* hv = nullptr;
        MCQ_REQUIRE(curandGetDirectionVectors32(&hv, CURAND_DIRECTION_VECTORS_32_JOEKUO6) ==
                        CURAND_STATUS_SUCCESS,
                    MCQ_ERR_INTERNAL, "curandGetDirectionVectors32 failed");
        MCQ_CUDA(cudaMemcpy(ptr, hv, kTableBytes, cudaMemcpyHostToDevice));
        int sms = 0;
        MCQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        g_sm_count[dev] = sms;
        g_scratch[dev] = static_cast<unsigned char*>(ptr);
        g_ctx_id[dev] = ctx;
    }
    *sm_count = g_sm_count[dev];
    return g_scratch[dev];
}
}  // namespace

static void qmc_pass_noalloc(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t salt_base,
                             int R, uint32_t offset, int64_t n_points, int flags, double* sums_device,
                             cudaStream_t stream) {
    MCQ_REQUIRE(m && p && sums_device, MCQ_ERR_INVALID, "model, payoff and sums_device must not be NULL");
    MCQ_REQUIRE(m->kind == MCQ_MODEL_GBM || m->kind == MCQ_MODEL_HESTON || m->kind == MCQ_MODEL_DUPIRE,
                MCQ_ERR_UNSUPPORTED, "the no-allocation pass takes GBM, Heston or parametric Dupire models");
    MCQ_REQUIRE(n_steps >= 1 && m->T > 0, MCQ_ERR_INVALID, "n_steps must be >= 1 and T > 0");
    const int D = n_steps * noise_dim(*m);
    MCQ_REQUIRE(D <= kMaxDims, MCQ_ERR_RANGE,
                "the no-allocation pass supports at most " + std::to_string(kMaxDims) +
                    " Sobol dimensions (steps x factors); got " + std::to_string(D));
    MCQ_REQUIRE(R >= 1 && R <= kMaxReplicas, MCQ_ERR_RANGE,
                "the no-allocation pass supports 1.." + std::to_string(kMaxReplicas) + " replicas; got " +
                    std::to_string(R));
    MCQ_REQUIRE(n_points >= 1 && (uint64_t)offset + (uint64_t)n_points <= (1ull << 32), MCQ_ERR_RANGE,
                "point range must be non-empty and end at or below 2^32");

    PassArgs a;
    a.m = m; a.p = p; a.n_steps = n_steps; a.gen = GEN_SOBOL; a.noise = NOISE_RAW; a.salt0 = salt_base;
    a.R = R; a.offset = offset; a.n_points = (uint64_t)n_points; a.flags = flags;
    Workspace unused;   // fill_params stages arrays only for basket / grid models, excluded above
    KParams k;
    fill_params(unused, a, k);

    // the kernel and work split of mcq_qmc_pass_device for this request (engine.cpp pass_async):
    // paths of at most 16 normals take the packed pass, whose items are whole tiles of 32 / D
    // groups; the plain pass otherwise (the assisted form it may choose for few long paths gives
    // the plain pass's bits)
    const void* fn = (D <= 16) ? lookup_sobol_packed(k.model, p->kind, false) : nullptr;
    const bool packed = fn != nullptr;
    // the plain pass in the launch variant the autotuner keeps for these families on a B200 (it does
    // not run here: no timing events on the caller's stream): the unrolled tile generator (all
    // variants give the same bits)
    if (!fn) fn = lookup_variant(GEN_SOBOL, NOISE_RAW, EST_PLAIN, k.model, p->kind, 2);
    if (!fn) fn = lookup_pass(GEN_SOBOL, NOISE_RAW, EST_PLAIN, k.model, p->kind, 0);
    MCQ_REQUIRE(fn != nullptr, MCQ_ERR_UNSUPPORTED, "no fused kernel for this model / payoff");
    const uint64_t g0 = a.offset >> 5;
    const uint64_t G = ((a.offset + a.n_points - 1) >> 5) - g0 + 1;
    uint64_t gpi = (G * (uint64_t)R + kTargetItems - 1) / kTargetItems;
    if (gpi < 1) gpi = 1;
    if (packed) {
        const uint64_t Q = (uint64_t)(32 / D);
        gpi = (gpi + Q - 1) / Q * Q;
    }
    const uint64_t ipr = (G + gpi - 1) / gpi;
    MCQ_REQUIRE(ipr * (uint64_t)R <= (uint64_t)kMaxItems, MCQ_ERR_RANGE,
                "work split needs more than " + std::to_string(kMaxItems) + " items");
    k.R = R; k.gpi = (int)gpi; k.items_per_rep = (int)ipr; k.n_items = (int)(ipr * R);
    k.offset = a.offset; k.n_points = a.n_points; k.g0 = g0; k.G = G;

    int sms = 0;
    unsigned char* base = scratch_for_current_device(&sms);
    const uint32_t* table = reinterpret_cast<const uint32_t*>(base);
    uint32_t* dirs = reinterpret_cast<uint32_t*>(base + kTableBytes);
    double* partials = reinterpret_cast<double*>(base + kTableBytes + kDirsBytes);
    k.dirs = dirs;
    k.partials = partials;

    size_t smem = (size_t)kWarpsPerBlock * 1024 * sizeof(float);
    int per_sm = 0;
    MCQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem));
    MCQ_REQUIRE(per_sm > 0, MCQ_ERR_INTERNAL, "kernel does not fit on an SM");
    // Sobol start words carried from group to group (one slot per 32-dimension tile), as the
    // allocating pass does: when items hold several groups, the slots stay within the default
    // 48 KB of dynamic shared memory (no attribute change) and keep the resident blocks per SM
    k.carry = 0;
    if (!packed && gpi >= 2) {
        const int words = 32 * ((D + 31) / 32);
        const size_t with = smem + (size_t)kWarpsPerBlock * words * sizeof(uint32_t);
        int per_sm_c = 0;
        if (with <= 48 * 1024) {
            MCQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_c, fn, kThreads, with));
            if (per_sm_c >= per_sm) {
                k.carry = words;
                smem = with;
            }
        }
    }
    long long blocks = ((long long)k.n_items + kWarpsPerBlock - 1) / kWarpsPerBlock;
    blocks = std::min<long long>(blocks, (long long)per_sm * sms);
    blocks = std::max<long long>(blocks, 1);

    launch_prescramble(table, salt_base, R, D, dirs, stream);
    void* args[] = {&k};
    MCQ_CUDA(cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(kThreads), args, smem, stream));
    launch_finalize(partials, R, k.items_per_rep, 2, sums_device, stream);
    MCQ_CUDA(cudaGetLastError());
}

}  // namespace mcq

extern "C" int mcq_qmc_pass_noalloc(const mcq_model* m, const mcq_payoff* p, int n_steps,
                                    uint32_t salt_base, int R, uint32_t offset, int64_t n_points,
                                    int flags, double* sums_device, void* stream) {
    try {
        mcq::qmc_pass_noalloc(m, p, n_steps, salt_base, R, offset, n_points, flags, sums_device,
                              (cudaStream_t)stream);
        return MCQ_OK;
    } catch (const mcq::Error& e) {
        mcq::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        mcq::set_last_error(e.what());
        return MCQ_ERR_INTERNAL;
    }
}
