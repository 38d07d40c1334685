// engine.h — host runtime of the pricing engine: device context, per-stream workspaces,
// BB/PCA handles, parameter translation and the fused-pass launcher.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <map>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/mcq.h"
#include "kparams.h"

namespace mcq {

// Errors cross the C ABI as status codes; inside the library they are exceptions.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MCQ_CUDA(call)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw ::mcq::Error(MCQ_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e_) + \
                                                 " at " __FILE__ ":" + std::to_string(__LINE__)); \
    } while (0)

#define MCQ_REQUIRE(cond, code, msg) \
    do { if (!(cond)) throw ::mcq::Error((code), (msg)); } while (0)

// Grow-only device / pinned-host buffers.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    void* ensure(size_t bytes);
    void release();
    ~DevBuf() { release(); }
};
struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    void* ensure(size_t bytes);
    void release();
    ~PinnedBuf() { release(); }
};

// Scratch owned by one stream: item partials, per-replica sums, scrambled direction words,
// small parameter uploads.  Launches on one workspace are ordered by its stream; a pass run on a
// caller's stream is joined back into it (`joined`, recorded on the caller's stream and waited
// on by the workspace stream), so later work on the workspace, and the read of its status word,
// comes after that pass.
struct Workspace {
    cudaStream_t stream = nullptr;
    cudaEvent_t joined = nullptr;
    DevBuf partials, sums, dirs, aux, dump, err;
    bool err_armed = false;   // err holds a fresh status from the last tensor-core pass
    PinnedBuf hsums, haux;
    DevBuf xbuf[8];       // long-lived scratch of the batched book (book.cu): kept across calls
    PinnedBuf xpin[2];
    DevBuf pca_z, pca_dw, pca_tmp;   // the large-N PCA route (pca_large.cu): fp16 normals, increments
    struct Blas {                    // its cuBLAS handle, created on first use
        void* h = nullptr;
        ~Blas();
    } blas;
    uint32_t dirs_salt0 = 0;
    int dirs_R = -1, dirs_D = -1;
    void ensure_stream();
    ~Workspace();
};

// BB / PCA handle (DeviceBBData / DevicePCAData, methods_cuda.cu:912-926).
struct Handle {
    int kind = 0;       // MCQ_NOISE_BB or MCQ_NOISE_PCA
    int n = 0;
    double T = 0;
    DevBuf table;       // BB: float4[N] + int2[N]; PCA: fp16 [m][m] row-major (row = output step)
    std::vector<float> host_f;   // BB: wl,wr,sd per dim; PCA: column-major float M
    std::vector<int> host_i;     // BB: m per dim
    // BB, N > 32: true when every window point of a level has the same (wl, wr, sd) in FP32 (a
    // uniform time grid); bb_lvl[u] is that triple for window level u = 0..4
    bool bb_uni = false;
    float bb_lvl[5][3] = {};
};

struct KernelInfo {
    int blocks_per_sm = 0;
    size_t smem = 0;
};

// Autotuner state of one kernel family with several compiled launch variants: the first large
// passes run one variant each, timed by events around the kernel on its own stream; the
// variant with the lower time per path-step is kept.  Variants compute identical sums, so
// tuning never changes a result.
inline constexpr int kMaxVariants = 3;
struct TuneState {
    int chosen = -1;
    bool done[kMaxVariants] = {};
    bool pending[kMaxVariants] = {};
    double per_unit[kMaxVariants] = {};
    double units[kMaxVariants] = {};
    cudaEvent_t ev[kMaxVariants][2] = {};
};

// Autotuner: the launch variant of family `key` (nvar variants) for a launch of `units` work;
// *trial set: record ev[variant][0] / [1] around the launch (engine.cpp).
int tune_pick(uint64_t key, int nvar, double units, double min_units, TuneState** trial);
const TuneState* tune_state(uint64_t key);   // nullptr until the family has been launched

struct Engine {
    std::mutex mu;
    bool ready = false;
    int device = -1;
    int sm_count = 148;
    uint32_t* d_dv = nullptr;                        // JoeKuo6 table [20000][32]
    std::vector<std::unique_ptr<Workspace>> pool;    // pool[0] is the default workspace
    int smem_optin = 227 * 1024;                     // dynamic shared memory a block may opt into
    std::map<std::pair<const void*, size_t>, KernelInfo> kinfo;   // occupancy per (kernel, smem)
    std::unordered_set<const void*> kattr;           // kernels whose smem limit is raised
    std::unordered_map<uint64_t, TuneState> tune;
    int launches = 0;                                // kernel launches issued (accounting)
    int last_gpi = 0, last_carry = 0;                // work layout of the last fused pass
    Workspace& ws(int i);
};

Engine& engine();
void ensure_ready(int device = -1);
void shutdown_engine();

// Everything a fused pass needs besides the geometry of the work.
struct PassArgs {
    const mcq_model* m = nullptr;
    const mcq_payoff* p = nullptr;
    int n_steps = 0;          // fine steps
    int est = EST_PLAIN;
    int M = 0;                // coupling factor (EST_COUPLED)
    bool level0 = false;      // coupled pass without a coarse path
    bool mlmc_h = false;      // h = (float)(T / n) as run_mlmc_cuda (else (float)T / n)
    int gen = GEN_SOBOL;
    int noise = NOISE_RAW;
    const Handle* bb = nullptr;
    const Handle* pca = nullptr;
    uint32_t salt0 = 42;
    int R = 1;
    uint64_t offset = 0;
    uint64_t n_points = 0;
    uint32_t seed = 0;
    uint32_t stream0 = 0;
    int flags = 0;
    float beta_cv = 0.f, E_ctrl = 0.f, z_star = 0.f;
    bool dump = false;
};

// Work items per pass are sized from the problem alone (never from the device) so that the
// split, and with it every sum, is the same on any GPU.  About eight items per resident warp of a
// B200 at four CTAs per SM: a warp's last item then costs at most an eighth of the pass (with
// three per warp the small first passes of the adaptive drivers lost up to a quarter).
inline constexpr long long kTargetItems = 148LL * 32 * 8;
// the adjoint's split: about eight items per resident warp (two CTAs of eight warps per SM)
inline constexpr long long kTargetItemsAdjoint = 148LL * 16 * 8;

int noise_dim(const mcq_model& m);
// KParams for a pass (make_params); basket / local-vol arrays are uploaded into ws.aux.
void fill_params(Workspace& ws, const PassArgs& a, KParams& k);
int nstat_of(int est);
int nstat_of(int est, int model_kind);   // basket levels carry per-asset deltas
// Enqueue one pass on ws.stream; d_out receives [R][nstat] doubles (device).
void pass_async(Workspace& ws, const PassArgs& a, double* d_out);
// Tensor-core PCA pass (N in {64, 128, 256}); called by pass_async.
void pca_pass_async(Workspace& ws, const PassArgs& a, KParams& k, double* d_out);
// PCA orderings the tensor-core pass does not hold (N > 32 outside {64, 128, 256}): fp16 normals,
// one library GEMM and the fused pass on the increments, batch by batch (pca_large.cu)
void pca_large_pass_async(Workspace& ws, const PassArgs& a, KParams& k, double* d_out);
// Enqueue, copy back and wait; returns [R][nstat].
std::vector<double> pass_sync(Workspace& ws, const PassArgs& a);
// After a synchronisation of ws.stream: raises MCQ_ERR_TIMEOUT if a bounded device-side wait of
// the workspace's last tensor-core or assisted pass gave up.
void check_err_word(Workspace& ws);
// Orders the workspace stream after everything issued so far on `caller`.
void join_caller_stream(Workspace& ws, cudaStream_t caller);
// The workspace's error word for a pass with bounded device waits (cleared unless it still holds
// an unread status of an earlier asynchronous pass).
int* arm_err_word(Workspace& ws);
// Occupancy / shared-memory set-up of a kernel for a dynamic shared-memory size (cached).
KernelInfo& kernel_info(const void* fn, size_t smem);
// Pathwise adjoint Greeks over R scrambled replicas (k_adjoint.cu).
void adjoint_run(const mcq_model& m, const mcq_payoff& p, int n_steps, uint32_t salt_base, int R,
                 uint64_t offset, uint64_t n_points, int flags, mcq_greeks& out, double* node_vega);
// Message returned by mcq_last_error() on this thread.
void set_last_error(const std::string& msg);
// Device capacity used by the reference's memory-derived batch sizing.
long long gpu_free_bytes_80();

}  // namespace mcq
