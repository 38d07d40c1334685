// engine.cpp — device context, workspaces, parameter translation and the pass launcher.
#include "engine.h"

#include <curand.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "adjoint.h"
#include "dispatch.h"
#include "pca.h"
#include "support.h"

namespace mcq {

// ------------------------------------------------------------------ buffers

void* DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return p;
    release();
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        throw Error(MCQ_ERR_NOMEM, "device allocation of " + std::to_string(want) + " bytes failed");
    }
    cap = want;
    return p;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}
void* PinnedBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return p;
    release();
    size_t want = std::max<size_t>(bytes, 256);
    if (cudaMallocHost(&p, want) != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        throw Error(MCQ_ERR_NOMEM, "pinned allocation failed");
    }
    cap = want;
    return p;
}
void PinnedBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

void Workspace::ensure_stream() {
    if (!stream) MCQ_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
}
Workspace::~Workspace() {
    if (joined) cudaEventDestroy(joined);
    if (stream) cudaStreamDestroy(stream);
}

void join_caller_stream(Workspace& ws, cudaStream_t caller) {
    if (!ws.joined) MCQ_CUDA(cudaEventCreateWithFlags(&ws.joined, cudaEventDisableTiming));
    MCQ_CUDA(cudaEventRecord(ws.joined, caller));
    MCQ_CUDA(cudaStreamWaitEvent(ws.stream, ws.joined, 0));
}

// ------------------------------------------------------------------ engine

Engine& engine() {
    static Engine e;
    return e;
}

Workspace& Engine::ws(int i) {
    while ((int)pool.size() <= i) pool.emplace_back(new Workspace());
    pool[i]->ensure_stream();
    return *pool[i];
}

void ensure_ready(int device) {
    Engine& E = engine();
    if (E.ready && (device < 0 || device == E.device)) return;
    if (E.ready) shutdown_engine();
    int dev = device;
    if (dev < 0) MCQ_CUDA(cudaGetDevice(&dev));
    MCQ_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    MCQ_CUDA(cudaGetDeviceProperties(&prop, dev));
    MCQ_REQUIRE(prop.major >= 10, MCQ_ERR_UNSUPPORTED,
                "this engine is built for sm_100a (B200); device " + std::string(prop.name) +
                    " is sm_" + std::to_string(prop.major) + std::to_string(prop.minor));
    E.device = dev;
    E.sm_count = prop.multiProcessorCount;
    E.smem_optin = (int)prop.sharedMemPerBlockOptin;
    // JoeKuo6 direction vectors, as ensure_sobol_dirvectors_uploaded (methods_cuda.cu:764-775).
    curandDirectionVectors32_t* hv = nullptr;
    MCQ_REQUIRE(curandGetDirectionVectors32(&hv, CURAND_DIRECTION_VECTORS_32_JOEKUO6) ==
                    CURAND_STATUS_SUCCESS,
                MCQ_ERR_INTERNAL, "curandGetDirectionVectors32 failed");
    MCQ_CUDA(cudaMalloc(&E.d_dv, sizeof(uint32_t) * 20000 * 32));
    MCQ_CUDA(cudaMemcpy(E.d_dv, hv, sizeof(uint32_t) * 20000 * 32, cudaMemcpyHostToDevice));
    E.ready = true;
}

void shutdown_engine() {
    Engine& E = engine();
    if (!E.ready) return;
    cudaDeviceSynchronize();
    E.pool.clear();
    E.kinfo.clear();
    for (auto& kv : E.tune)
        for (auto& pr : kv.second.ev)
            for (auto& ev : pr)
                if (ev) cudaEventDestroy(ev);
    E.tune.clear();
    if (E.d_dv) cudaFree(E.d_dv);
    E.d_dv = nullptr;
    E.ready = false;
}

long long gpu_free_bytes_80() {   // gpu_free_bytes, methods_cuda.cu:258-263
    size_t f = 0, t = 0;
    MCQ_CUDA(cudaMemGetInfo(&f, &t));
    return (long long)((double)f * 0.8);
}

// ------------------------------------------------------------------ parameter translation

int noise_dim(const mcq_model& m) {   // model_noise_dim, models.hpp:78-87
    switch (m.kind) {
        case MCQ_MODEL_HESTON: return 2;
        case MCQ_MODEL_MULTI_DUPIRE:
        case MCQ_MODEL_BASKET_GBM: return m.n_assets;
        default: return 1;
    }
}

int nstat_of(int est, int model) {
    if (est == EST_COUPLED && (model == MCQ_MODEL_BASKET_GBM || model == MCQ_MODEL_MULTI_DUPIRE)) return 4 + kMaxBasket;
    return nstat_of(est);
}

int nstat_of(int est) {
    switch (est) {
        case EST_COUPLED: return 4;
        case EST_CV_ASIAN:
        case EST_CV_DUPIRE: return 7;
        default: return 2;
    }
}

static int model_code(int kind) {
    switch (kind) {
        case MCQ_MODEL_GBM: return MOD_GBM;
        case MCQ_MODEL_HESTON: return MOD_HESTON;
        case MCQ_MODEL_DUPIRE: return MOD_DUPIRE;
        case MCQ_MODEL_MULTI_DUPIRE: return MOD_MULTI;
        case MCQ_MODEL_LOCALVOL_GRID: return MOD_LVGRID;
        case MCQ_MODEL_BASKET_GBM: return MOD_BASKET;
    }
    throw Error(MCQ_ERR_INVALID, "unknown model kind " + std::to_string(kind));
}

static bool is_pow2(long long x) { return x > 0 && (x & (x - 1)) == 0; }

static bool uniform_axis(const double* a, int n, double* a0, double* inv_d) {
    if (!a || n < 2) return false;
    double d = (a[n - 1] - a[0]) / (n - 1);
    if (!(d > 0)) return false;
    for (int i = 0; i < n; i++)
        if (std::fabs(a[i] - (a[0] + d * i)) > 1e-9 * std::max(1.0, std::fabs(a[i]))) return false;
    *a0 = a[0];
    *inv_d = 1.0 / d;
    return true;
}

// make_params (methods_cuda.cu:986-1053) in the engine's layout; aux arrays are staged in `ws`.
void fill_params(Workspace& ws, const PassArgs& a, KParams& k) {
    const mcq_model& m = *a.m;
    const mcq_payoff& p = *a.p;
    std::memset(&k, 0, sizeof(k));
    k.gen = a.gen;
    k.noise = a.noise;
    k.model = model_code(m.kind);
    k.payoff = p.kind;
    k.est = a.est;
    k.n_steps = a.n_steps;
    k.d_noise = noise_dim(m);
    k.D = a.n_steps * k.d_noise;
    k.dstride = k.D;
    k.flags = a.flags;
    k.nstat = nstat_of(a.est, m.kind);

    const float Tf = (float)m.T;
    const float h = a.mlmc_h ? (float)(m.T / a.n_steps) : Tf / (float)a.n_steps;
    k.T = Tf;
    k.h = h;
    k.sqrt_h = sqrtf(h);
    k.S0 = (float)m.S0;
    k.inv_S0 = 1.0f / k.S0;
    k.mu = (float)m.mu;
    k.sigma = (float)m.sigma;
    k.kappa = (float)m.kappa;
    k.theta = (float)m.theta;
    k.xi = (float)m.xi;
    k.v0 = (float)m.v0;
    k.L10 = (float)m.hes_L10;
    k.L11 = (float)m.hes_L11;
    // 1 - e^{-kappa h} with its own relative precision: at fine levels e^{-kappa h} lies within a few
    // FP32 ulps of 1, and rounding it there biases the mean reversion by up to 0.4 % at 2^18 steps
    // (the reference rounds expf(-kappa h) itself, methods_cuda.cu:282)
    k.om_f = (float)(-std::expm1(-(double)k.kappa * (double)h));
    k.sigma0 = (float)m.sigma0;
    k.alpha = (float)m.alpha;
    k.bm1 = (float)m.beta_d - 1.0f;
    if (m.kind == MCQ_MODEL_DUPIRE) k.sigma = k.sigma0;   // :1041 sigma_eff for the GBM control

    if (a.est == EST_COUPLED) {
        k.M = a.M;
        k.n_coarse = a.level0 ? 0 : a.n_steps / a.M;
        k.hc = (float)(m.T / std::max(k.n_coarse, 1));
        k.om_c = (float)(-std::expm1(-(double)k.kappa * (double)k.hc));
        if (a.level0) k.M = INT_MAX;   // the coarse path never steps on level 0
    }
    if (m.kind == MCQ_MODEL_HESTON && (a.flags & MCQ_FLAG_HESTON_MILSTEIN)) {
        k.mil = 0.25f * k.xi * k.xi;
    }

    k.K = (float)p.K;
    k.B = (float)p.B;
    k.pay_T = (float)p.T;
    switch (p.kind) {
        case MCQ_PAYOFF_EUROPEAN:
        case MCQ_PAYOFF_BARRIER_UP_OUT:
        case MCQ_PAYOFF_BARRIER_DOWN_OUT:
        case MCQ_PAYOFF_BASKET: k.disc = (float)std::exp(-p.r * p.T); break;
        default: k.disc = 1.0f;
    }
    if (p.kind == MCQ_PAYOFF_LOOKBACK || p.kind == MCQ_PAYOFF_BARRIER_UP_OUT ||
        p.kind == MCQ_PAYOFF_BARRIER_DOWN_OUT) {   // d_apply_bgk, :326-331
        const float sb = (float)p.sigma;
        k.corr_f = (float)std::exp((double)(-0.5826f * sb * sqrtf(h)));
        k.corr_c = (float)std::exp((double)(-0.5826f * sb * sqrtf(k.hc > 0 ? k.hc : h)));
    } else {
        k.corr_f = k.corr_c = 1.0f;
    }
    k.u_cap = (a.flags & MCQ_FLAG_COMPAT_U_INF) ? 1.0f : 0x1.fffffep-1f;
    k.beta_cv = a.beta_cv;
    k.E_ctrl = a.E_ctrl;
    k.z_star = a.z_star;
    k.ctrl_sigma = k.sigma0;
    k.seed = a.seed;
    k.stream_base = a.stream0;

    // multi-asset parameters
    if (m.kind == MCQ_MODEL_MULTI_DUPIRE || m.kind == MCQ_MODEL_BASKET_GBM) {
        const int n = m.n_assets;
        MCQ_REQUIRE(n >= 1, MCQ_ERR_INVALID, "basket needs n_assets >= 1");
        MCQ_REQUIRE(n <= kMaxHugeBasket, MCQ_ERR_UNSUPPORTED,
                    "basket width " + std::to_string(n) + " exceeds the limit of " + std::to_string(kMaxHugeBasket) +
                        " assets");
        MCQ_REQUIRE(m.S0_vec != nullptr, MCQ_ERR_INVALID, "basket needs S0_vec");
        if (m.kind == MCQ_MODEL_BASKET_GBM)
            MCQ_REQUIRE(m.sigma_vec != nullptr, MCQ_ERR_INVALID, "basket needs sigma_vec");
        std::vector<float> pk((size_t)3 * n + (size_t)n * n, 0.f);
        // the second block: per-asset sigma for the GBM basket; for the Dupire basket the inverse
        // of the S0 that scales the asset's local volatility (asset 0's, as the reference, or
        // its own under MCQ_FLAG_BASKET_OWN_S0)
        const bool own = (a.flags & MCQ_FLAG_BASKET_OWN_S0) != 0;
        for (int i = 0; i < n; i++) {
            pk[i] = (float)m.S0_vec[i];
            if (m.kind == MCQ_MODEL_MULTI_DUPIRE) pk[n + i] = 1.0f / (float)m.S0_vec[own ? i : 0];
            else pk[n + i] = m.sigma_vec ? (float)m.sigma_vec[i] : 0.f;
            pk[2 * n + i] = m.weights ? (float)m.weights[i] : 1.0f / n;
        }
        const bool unc = m.uncorrelated || !m.L;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                pk[3 * n + i * n + j] = unc ? (i == j ? 1.f : 0.f) : (float)m.L[i * n + j];
        k.n_assets = n;
        k.uncorrelated = unc ? 1 : 0;
        k.inv_S0 = 1.0f / (float)m.S0_vec[0];     // c_p.S0 = S0[0] (:1046)
        k.S0 = (float)m.S0_vec[0];
        float* d = (float*)ws.aux.ensure(pk.size() * sizeof(float));
        MCQ_CUDA(cudaMemcpyAsync(d, pk.data(), pk.size() * sizeof(float), cudaMemcpyHostToDevice, ws.stream));
        k.bsk = d;
    }
    if (m.kind == MCQ_MODEL_LOCALVOL_GRID) {
        double K0, iK, t0, it;
        MCQ_REQUIRE(uniform_axis(m.lv_K, m.lv_nK, &K0, &iK) && uniform_axis(m.lv_t, m.lv_nt, &t0, &it),
                    MCQ_ERR_UNSUPPORTED, "local-vol grid axes must be uniform with >= 2 nodes");
        MCQ_REQUIRE(m.lv_sigma != nullptr, MCQ_ERR_INVALID, "local-vol grid needs lv_sigma");
        const size_t nn = (size_t)m.lv_nK * m.lv_nt;
        std::vector<float> g(nn);
        for (size_t i = 0; i < nn; i++) g[i] = (float)m.lv_sigma[i];
        // the grid, then the time rows of the pass's fine steps (16-byte aligned)
        const size_t grid_bytes = (nn * sizeof(float) + 15) & ~(size_t)15;
        const int n_rows = a.n_steps + 1;
        char* d = (char*)ws.aux.ensure(grid_bytes + (size_t)n_rows * sizeof(float2));
        MCQ_CUDA(cudaMemcpyAsync(d, g.data(), nn * sizeof(float), cudaMemcpyHostToDevice, ws.stream));
        k.lv = (const float*)d;
        k.lv_nK = m.lv_nK;
        k.lv_nt = m.lv_nt;
        k.lv_K0 = (float)K0;
        k.lv_inv_dK = (float)iK;
        k.lv_t0 = (float)t0;
        k.lv_inv_dt = (float)it;
        float2* rows = (float2*)(d + grid_bytes);
        launch_lv_rows(k, rows, n_rows, ws.stream);
        engine().launches++;
        k.lv_rows = rows;
    }
}

// ------------------------------------------------------------------ launcher


// Resident blocks per SM of kernel `fn` at `smem` bytes of dynamic shared memory (kThreads
// threads).  A kernel's dynamic shared-memory limit is raised to the device's opt-in maximum
// once, so that occupancy can be asked for several sizes (with and without carry slots) and any
// of them launched.
KernelInfo& kernel_info(const void* fn, size_t smem) {
    Engine& E = engine();
    const auto key = std::make_pair(fn, smem);
    auto it = E.kinfo.find(key);
    if (it != E.kinfo.end()) return it->second;
    MCQ_REQUIRE(smem <= (size_t)E.smem_optin, MCQ_ERR_INTERNAL, "kernel shared memory above the device limit");
    if (!E.kattr.count(fn)) {
        MCQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, E.smem_optin));
        E.kattr.insert(fn);
    }
    KernelInfo ki;
    ki.smem = smem;
    MCQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ki.blocks_per_sm, fn, kThreads, smem));
    MCQ_REQUIRE(ki.blocks_per_sm > 0, MCQ_ERR_INTERNAL, "kernel does not fit on an SM");
    return E.kinfo[key] = ki;
}

// The autotuner.  A family of kernels compiled with nvar launch variants that differ only in
// register allocation, scheduling or work granularity inside a launch (never in arithmetic, so
// every variant gives the same bits) is tuned once per process: its first launches of at least
// min_units work units run one variant each, timed with events on the launching stream (the
// caller records them around its launch when *trial is set), and the variant with the least time
// per unit is kept.  MCQ_TUNE=<v> forces variant v.
int tune_pick(uint64_t key, int nvar, double units, double min_units, TuneState** trial) {
    Engine& E = engine();
    *trial = nullptr;
    if (nvar <= 1) return 0;
    if (const char* force = std::getenv("MCQ_TUNE")) return std::min(std::max(std::atoi(force), 0), nvar - 1);
    TuneState& ts = E.tune[key];
    for (int v = 0; v < nvar; v++) {
        if (ts.pending[v]) {
            float ms = 0.f;
            MCQ_CUDA(cudaEventSynchronize(ts.ev[v][1]));
            MCQ_CUDA(cudaEventElapsedTime(&ms, ts.ev[v][0], ts.ev[v][1]));
            ts.per_unit[v] = ms / ts.units[v];
            ts.pending[v] = false;
            ts.done[v] = true;
        }
    }
    int first_untried = -1;
    for (int v = 0; v < nvar; v++)
        if (!ts.done[v] && first_untried < 0) first_untried = v;
    if (ts.chosen < 0 && first_untried < 0) {
        ts.chosen = 0;
        for (int v = 1; v < nvar; v++)
            if (ts.per_unit[v] < ts.per_unit[ts.chosen]) ts.chosen = v;
    }
    if (ts.chosen >= 0) return ts.chosen;
    if (units < min_units || ts.pending[first_untried]) return 0;
    const int v = first_untried;
    if (!ts.ev[v][0]) {
        MCQ_CUDA(cudaEventCreate(&ts.ev[v][0]));
        MCQ_CUDA(cudaEventCreate(&ts.ev[v][1]));
    }
    ts.units[v] = units;
    ts.pending[v] = true;
    *trial = &ts;
    return v;
}

const TuneState* tune_state(uint64_t key) {
    auto it = engine().tune.find(key);
    return it == engine().tune.end() ? nullptr : &it->second;
}

void pass_async(Workspace& ws, const PassArgs& a, double* d_out) {
    Engine& E = engine();
    MCQ_REQUIRE(a.m && a.p, MCQ_ERR_INVALID, "null model or payoff");
    MCQ_REQUIRE(a.n_steps >= 1, MCQ_ERR_INVALID, "n_steps must be >= 1");
    MCQ_REQUIRE(a.R >= 1, MCQ_ERR_INVALID, "R must be >= 1");
    MCQ_REQUIRE(a.m->T > 0, MCQ_ERR_INVALID, "T must be > 0");
    if (a.n_points == 0) {
        MCQ_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * a.R * nstat_of(a.est, a.m->kind), ws.stream));
        return;
    }
    KParams k;
    fill_params(ws, a, k);
    const int D = k.D;
    int nb = 0;
    if (k.model == MOD_MULTI || k.model == MOD_BASKET) nb = k.n_assets;

    if (a.gen == GEN_SOBOL) {
        MCQ_REQUIRE(D <= 20000, MCQ_ERR_RANGE,
                    "Sobol dimension " + std::to_string(D) + " exceeds the direction table (20000)");
        MCQ_REQUIRE(a.offset + a.n_points <= (1ull << 32), MCQ_ERR_RANGE,
                    "Sobol point index beyond 2^32 (offset " + std::to_string(a.offset) + " + " +
                        std::to_string(a.n_points) + ")");
    }
    if (a.noise == NOISE_BB) {
        MCQ_REQUIRE(k.d_noise == 1, MCQ_ERR_UNSUPPORTED, "Brownian bridge needs a one-factor model");
        MCQ_REQUIRE(a.bb && a.bb->kind == MCQ_NOISE_BB && a.bb->n == a.n_steps, MCQ_ERR_INVALID,
                    "Brownian-bridge handle missing or built for a different step count");
        MCQ_REQUIRE(a.gen == GEN_SOBOL, MCQ_ERR_UNSUPPORTED, "Brownian bridge is a QMC transform");
        k.bb = (const float4*)a.bb->table.p;
        k.bbi = (const int2*)((const float4*)a.bb->table.p + a.n_steps);
        if (a.bb->bb_uni) std::memcpy(k.bbw, a.bb->bb_lvl, sizeof(k.bbw));
    }
    // the kernel family: the bridge with uniform window weights reads them from the parameters
    const int knoise = (a.noise == NOISE_BB && D > 32 && a.bb->bb_uni) ? NOISE_BB_UNI : a.noise;
    const bool pca_tc = (a.noise == NOISE_PCA) && (D == 64 || D == 128 || D == 256);
    if (a.noise == NOISE_PCA) {
        MCQ_REQUIRE(k.d_noise == 1, MCQ_ERR_UNSUPPORTED, "PCA needs a one-factor model");
        MCQ_REQUIRE(a.gen == GEN_SOBOL, MCQ_ERR_UNSUPPORTED, "PCA is a QMC transform");
        MCQ_REQUIRE(a.pca && a.pca->kind == MCQ_NOISE_PCA && a.pca->n == a.n_steps, MCQ_ERR_INVALID,
                    "PCA handle missing or built for a different step count");
        k.pca = a.pca->table.p;
    }
    // fused: N <= 32 inside k_pass, N in {64, 128, 256} in the tensor-core pass (its factor in
    // shared memory); other N through fp16 normals, a library GEMM and the pass on increments
    if (a.noise == NOISE_PCA && D > 32 && D != 64 && D != 128 && D != 256 && !a.dump) {
        pca_large_pass_async(ws, a, k, d_out);
        return;
    }
    MCQ_REQUIRE(!(a.noise == NOISE_PCA && a.dump) || D <= 32 || D == 64 || D == 128 || D == 256,
                MCQ_ERR_UNSUPPORTED, "the PCA dump probe covers N <= 32 and N in {64, 128, 256}");
    if (pca_tc) {
        pca_pass_async(ws, a, k, d_out);
        return;
    }

    const void* fn = a.dump ? lookup_misc(a.gen, a.noise, a.est, k.model, nb, true)
                            : lookup_pass(a.gen, knoise, a.est, k.model, a.p->kind, nb);
    // short raw-ordered Sobol paths: 32 / D path groups per tile instead of one
    const void* packed = nullptr;
    if (!a.dump && a.gen == GEN_SOBOL && a.noise == NOISE_RAW && D <= 16 &&
        (a.est == EST_PLAIN || a.est == EST_COUPLED))
        packed = lookup_sobol_packed(k.model, a.p->kind, a.est == EST_COUPLED);
    if (packed) fn = packed;
    // few, long raw-ordered paths (fewer 32-path groups than 8 warps per SM, at least 256 normals
    // a path): helper warps generate each path-owning warp's normals.  Measured on 512 groups:
    // 1.1-2x faster from 256 normals up, slower below 128 (the ring's handoffs cost more than
    // the generation they hide)
    const void* assist = nullptr;
    if (!a.dump && !packed && a.noise == NOISE_RAW && D >= 256 && (a.est == EST_PLAIN || a.est == EST_COUPLED)) {
        const uint64_t groups = (((a.offset + a.n_points - 1) >> 5) - (a.offset >> 5) + 1) * (uint64_t)a.R;
        if (groups < (uint64_t)E.sm_count * 8)
            assist = lookup_assist(a.gen, k.model, a.p->kind, a.est == EST_COUPLED);
    }
    if (assist) fn = assist;
    // launch variant: MCQ_TUNE=<v> forces one; otherwise the autotuner picks per family
    int variant = 0;
    TuneState* trial = nullptr;
    const int nvar = (a.dump || packed || assist) ? 1 : n_variants(a.gen, knoise, a.est, k.model);
    if (nvar > 1) {
        const uint64_t key = (uint64_t)a.gen | ((uint64_t)knoise << 4) | ((uint64_t)a.est << 8) |
                             ((uint64_t)k.model << 12) | ((uint64_t)a.p->kind << 16);
        variant = tune_pick(key, nvar, (double)a.R * (double)a.n_points * (double)k.D, (double)(1 << 26), &trial);
        if (variant > 0) fn = lookup_variant(a.gen, knoise, a.est, k.model, a.p->kind, variant);
    }
    MCQ_REQUIRE(fn != nullptr, MCQ_ERR_UNSUPPORTED,
                "no fused kernel for gen " + std::to_string(a.gen) + " noise " + std::to_string(a.noise) +
                    " est " + std::to_string(a.est) + " model " + std::to_string(a.m->kind) + " payoff " +
                    std::to_string(a.p->kind));

    // work split: 32-point groups, `gpi` groups per item, items per replica
    const uint64_t g0 = a.offset >> 5;
    const uint64_t G = ((a.offset + a.n_points - 1) >> 5) - g0 + 1;
    uint64_t gpi = (G * (uint64_t)a.R + kTargetItems - 1) / kTargetItems;
    if (gpi < 1) gpi = 1;
    if (packed) {   // whole tiles of 32 / D groups per item
        const uint64_t Q = (uint64_t)(32 / D);
        gpi = (gpi + Q - 1) / Q * Q;
    }
    const uint64_t ipr = (G + gpi - 1) / gpi;
    MCQ_REQUIRE(ipr * (uint64_t)a.R < (1ull << 31), MCQ_ERR_RANGE, "too many work items");
    k.R = a.R;
    k.gpi = (int)gpi;
    k.items_per_rep = (int)ipr;
    k.n_items = (int)(ipr * a.R);
    k.offset = a.offset;
    k.n_points = a.n_points;
    k.g0 = g0;
    k.G = G;

    if (a.gen == GEN_SOBOL) {
        if (!(ws.dirs_salt0 == a.salt0 && ws.dirs_R == a.R && ws.dirs_D == D)) {
            uint32_t* d = (uint32_t*)ws.dirs.ensure(sizeof(uint32_t) * (size_t)a.R * 33 * D);
            launch_prescramble(E.d_dv, a.salt0, a.R, D, d, ws.stream);
            E.launches++;
            ws.dirs_salt0 = a.salt0;
            ws.dirs_R = a.R;
            ws.dirs_D = D;
        }
        k.dirs = (const uint32_t*)ws.dirs.p;
    }
    const int nst = a.dump ? 1 : k.nstat;
    k.nstat = nst;
    k.partials = (double*)ws.partials.ensure(sizeof(double) * (size_t)k.n_items * nst);
    if (a.dump) {
        k.dump = (float*)ws.dump.ensure(sizeof(float) * (size_t)a.R * a.n_points * D);
    }

    const int skel = (a.noise == NOISE_BB && D > 32) ? ((D >> 5) + 1) * 32 : 0;
    const int accf = (!a.dump && a.est == EST_COUPLED && (k.model == MOD_BASKET || k.model == MOD_MULTI))
                         ? ((2 * nst + 3) & ~3) : 0;
    size_t smem = assist ? (size_t)kAssistTeams * kAssistTeamBytes
                         : (size_t)kWarpsPerBlock * (1024 + skel + accf) * sizeof(float);
    // Sobol start words carried from group to group of an item (one slot per tile a group
    // generates): kept when an item has several groups and the slots leave the kernel's resident
    // blocks per SM unchanged
    k.carry = 0;
    if (a.gen == GEN_SOBOL && !assist && !packed && gpi >= 2) {
        int tiles = 0;
        if (a.noise == NOISE_RAW) tiles = (D + 31) / 32;
        else if ((a.noise == NOISE_BB || a.noise == NOISE_BB_UNI) && D > 32) tiles = ((D >> 5) + 31) / 32 + (D >> 5);
        else if (a.noise == NOISE_BB || a.noise == NOISE_BB_UNI || knoise == NOISE_PCA) tiles = 1;
        const size_t with = smem + (size_t)kWarpsPerBlock * 32 * tiles * sizeof(uint32_t);
        if (tiles > 0 && with <= (size_t)E.smem_optin &&
            kernel_info(fn, with).blocks_per_sm >= kernel_info(fn, smem).blocks_per_sm) {
            k.carry = 32 * tiles;
            smem = with;
        }
    }
    KernelInfo& ki = kernel_info(fn, smem);
    E.last_gpi = k.gpi;
    E.last_carry = k.carry;
    const int items_per_block = assist ? kAssistTeams : kWarpsPerBlock;
    long long blocks = ((long long)k.n_items + items_per_block - 1) / items_per_block;
    blocks = std::min<long long>(blocks, (long long)ki.blocks_per_sm * E.sm_count);
    blocks = std::max<long long>(blocks, 1);
    if (assist) k.err = arm_err_word(ws);
    void* args[] = {&k};
    if (trial) MCQ_CUDA(cudaEventRecord(trial->ev[variant][0], ws.stream));
    MCQ_CUDA(cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(kThreads), args, smem, ws.stream));
    if (trial) MCQ_CUDA(cudaEventRecord(trial->ev[variant][1], ws.stream));
    launch_finalize(k.partials, a.R, k.items_per_rep, nst, d_out, ws.stream);
    E.launches += 2;
    MCQ_CUDA(cudaGetLastError());
}

// Tensor-core PCA pass: CTA work items are runs of 256-path tiles of one replica; each item
// leaves one record per warp, reduced per replica by k_finalize.
void pca_pass_async(Workspace& ws, const PassArgs& a, KParams& k, double* d_out) {
    Engine& E = engine();
    const int N = k.D;
    const void* fn = lookup_pca(k.model, a.p->kind, a.est == EST_COUPLED, a.dump);
    MCQ_REQUIRE(fn != nullptr, MCQ_ERR_UNSUPPORTED, "no tensor-core PCA kernel for this model / payoff");
    const uint64_t g0 = a.offset >> 5;
    const uint64_t G = ((a.offset + a.n_points - 1) >> 5) - g0 + 1;
    const uint64_t gpt = (uint64_t)pca_tile_paths() / 32;   // 32-point groups per tile
    const uint64_t tiles = (G + gpt - 1) / gpt;
    // about 32 items per CTA (one CTA per SM): with four, the CTA that drew a fifth item set the
    // kernel's length (a fifth of the pass idle at the tail)
    const uint64_t target = 148ULL * 32;
    uint64_t tpi = (tiles * (uint64_t)a.R + target - 1) / target;
    if (tpi < 1) tpi = 1;
    const uint64_t ipr = (tiles + tpi - 1) / tpi;
    MCQ_REQUIRE(ipr * (uint64_t)a.R * pca_warps() < (1ull << 31), MCQ_ERR_RANGE, "too many work items");
    k.R = a.R;
    k.gpi = (int)tpi;
    k.items_per_rep = (int)ipr;
    k.n_items = (int)(ipr * a.R);
    k.offset = a.offset;
    k.n_points = a.n_points;
    k.g0 = g0;
    k.G = G;
    if (!(ws.dirs_salt0 == a.salt0 && ws.dirs_R == a.R && ws.dirs_D == N)) {
        uint32_t* d = (uint32_t*)ws.dirs.ensure(sizeof(uint32_t) * (size_t)a.R * 33 * N);
        launch_prescramble(E.d_dv, a.salt0, a.R, N, d, ws.stream);
        E.launches++;
        ws.dirs_salt0 = a.salt0;
        ws.dirs_R = a.R;
        ws.dirs_D = N;
    }
    k.dirs = (const uint32_t*)ws.dirs.p;
    const int nst = a.dump ? 1 : k.nstat;
    k.nstat = nst;
    k.partials = (double*)ws.partials.ensure(sizeof(double) * (size_t)k.n_items * pca_warps() * nst);
    if (a.dump) k.dump = (float*)ws.dump.ensure(sizeof(float) * (size_t)a.R * a.n_points * N);
    k.err = arm_err_word(ws);
    const size_t smem = pca_smem_bytes(N);
    int per_sm = 0;
    MCQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MCQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, pca_threads(), smem));
    MCQ_REQUIRE(per_sm > 0, MCQ_ERR_INTERNAL, "PCA kernel does not fit on an SM");
    long long blocks = std::min<long long>((long long)k.n_items, (long long)per_sm * E.sm_count);
    blocks = std::max<long long>(blocks, 1);
    void* args[] = {&k};
    MCQ_CUDA(cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(pca_threads()), args, smem, ws.stream));
    launch_finalize(k.partials, a.R, k.items_per_rep * pca_warps(), nst, d_out, ws.stream);
    E.launches += 2;
    MCQ_CUDA(cudaGetLastError());
}

// A bounded device wait that gave up leaves MCQ_ERR_TIMEOUT in the workspace's error word.  The
// word is cleared only when it is armed afresh after a check, so a failure of an asynchronous pass
// stays there until the next synchronous call on the workspace reads it.
int* arm_err_word(Workspace& ws) {
    int* err = (int*)ws.err.ensure(sizeof(int));
    if (!ws.err_armed) {
        MCQ_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ws.stream));
        ws.err_armed = true;
    }
    return err;
}

void check_err_word(Workspace& ws) {
    if (!ws.err_armed) return;
    // read on the workspace stream, which a pass on a caller's stream has been joined into
    // (join_caller_stream), so the word is read after every pass that may have set it
    int* h = (int*)ws.haux.ensure(sizeof(int));
    MCQ_CUDA(cudaMemcpyAsync(h, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, ws.stream));
    MCQ_CUDA(cudaStreamSynchronize(ws.stream));
    ws.err_armed = false;
    MCQ_REQUIRE(*h == 0, MCQ_ERR_TIMEOUT, "a bounded device-side wait timed out (status " + std::to_string(*h) + ")");
}

std::vector<double> pass_sync(Workspace& ws, const PassArgs& a) {
    const size_t n = (size_t)a.R * (a.dump ? 1 : nstat_of(a.est, a.m->kind));
    double* d = (double*)ws.sums.ensure(sizeof(double) * n);
    pass_async(ws, a, d);
    double* h = (double*)ws.hsums.ensure(sizeof(double) * n);
    MCQ_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost, ws.stream));
    MCQ_CUDA(cudaStreamSynchronize(ws.stream));
    check_err_word(ws);
    return std::vector<double>(h, h + n);
}

}  // namespace mcq

namespace mcq {

// ------------------------------------------------------------------ adjoint Greeks

void adjoint_run(const mcq_model& m, const mcq_payoff& p, int n_steps, uint32_t salt_base, int R,
                 uint64_t offset, uint64_t n_points, int flags, mcq_greeks& out, double* node_vega) {
    Engine& E = engine();
    MCQ_REQUIRE(m.kind == MCQ_MODEL_GBM || m.kind == MCQ_MODEL_DUPIRE || m.kind == MCQ_MODEL_LOCALVOL_GRID ||
                    m.kind == MCQ_MODEL_HESTON,
                MCQ_ERR_UNSUPPORTED, "adjoint Greeks: GBM, Heston, parametric Dupire or grid local-vol models");
    MCQ_REQUIRE(p.kind == MCQ_PAYOFF_EUROPEAN || p.kind == MCQ_PAYOFF_ASIAN || p.kind == MCQ_PAYOFF_LOOKBACK,
                MCQ_ERR_UNSUPPORTED, "adjoint Greeks: European, Asian or lookback payoffs (Lipschitz)");
    if (m.kind == MCQ_MODEL_HESTON)
        MCQ_REQUIRE(n_steps >= 16 && n_steps % 16 == 0 && n_steps <= 1024, MCQ_ERR_UNSUPPORTED,
                    "adjoint Greeks (Heston): n_steps must be a multiple of 16 in [16, 1024]");
    else
        MCQ_REQUIRE(n_steps >= 32 && n_steps % 32 == 0 && n_steps <= 1024, MCQ_ERR_UNSUPPORTED,
                    "adjoint Greeks: n_steps must be a multiple of 32 in [32, 1024]");
    MCQ_REQUIRE(R >= 1 && n_points >= 1 && offset + n_points <= (1ull << 32), MCQ_ERR_RANGE, "bad replica / point range");
    auto t0 = std::chrono::steady_clock::now();
    const int l0 = E.launches;
    Workspace& ws = E.ws(0);
    PassArgs a;
    a.m = &m; a.p = &p; a.n_steps = n_steps; a.gen = GEN_SOBOL; a.salt0 = salt_base; a.R = R;
    a.offset = offset; a.n_points = n_points; a.flags = flags;
    KParams k;
    fill_params(ws, a, k);
    const int n_nodes = (m.kind == MCQ_MODEL_LOCALVOL_GRID) ? m.lv_nK * m.lv_nt : 0;
    MCQ_REQUIRE(n_nodes <= 4096, MCQ_ERR_UNSUPPORTED, "adjoint Greeks: at most 4096 grid nodes");
    // the checkpoint interval is a launch variant (same bits); variants whose shared memory does
    // not fit one CTA per SM are left out
    int nvar = adjoint_variants(k.model);
    while (nvar > 1 && adjoint_smem_bytes(k.model, n_steps, n_nodes, nvar - 1) > 227 * 1024) nvar--;
    TuneState* trial = nullptr;
    const uint64_t key = (1ULL << 40) | ((uint64_t)k.model << 4) | (uint64_t)p.kind;
    const int variant = tune_pick(key, nvar, (double)R * (double)n_points * (double)n_steps, (double)(1 << 26), &trial);
    const void* fn = lookup_adjoint(k.model, p.kind, variant);
    MCQ_REQUIRE(fn != nullptr, MCQ_ERR_UNSUPPORTED, "no adjoint kernel for this model / payoff");
    const uint64_t g0 = offset >> 5;
    const uint64_t G = ((offset + n_points - 1) >> 5) - g0 + 1;
    const long long target = kTargetItemsAdjoint;
    uint64_t gpi = (G * (uint64_t)R + target - 1) / target;
    if (gpi < 1) gpi = 1;
    const uint64_t ipr = (G + gpi - 1) / gpi;
    k.R = R; k.gpi = (int)gpi; k.items_per_rep = (int)ipr; k.n_items = (int)(ipr * R);
    k.offset = offset; k.n_points = n_points; k.g0 = g0; k.G = G;
    if (!(ws.dirs_salt0 == salt_base && ws.dirs_R == R && ws.dirs_D == k.D)) {
        uint32_t* d = (uint32_t*)ws.dirs.ensure(sizeof(uint32_t) * (size_t)R * 33 * k.D);
        launch_prescramble(E.d_dv, salt_base, R, k.D, d, ws.stream);
        E.launches++;
        ws.dirs_salt0 = salt_base; ws.dirs_R = R; ws.dirs_D = k.D;
    }
    k.dirs = (const uint32_t*)ws.dirs.p;
    k.nstat = 4;
    k.partials = (double*)ws.partials.ensure(sizeof(double) * (size_t)k.n_items * 4);
    double* d_nodes = nullptr;
    if (n_nodes) {
        d_nodes = (double*)ws.dump.ensure(sizeof(double) * n_nodes);
        MCQ_CUDA(cudaMemsetAsync(d_nodes, 0, sizeof(double) * n_nodes, ws.stream));
    }
    k.node_out = d_nodes;
    const size_t smem = adjoint_smem_bytes(k.model, n_steps, n_nodes, variant);
    KernelInfo& ki = kernel_info(fn, smem);
    long long blocks = std::min<long long>(((long long)k.n_items + kWarpsPerBlock - 1) / kWarpsPerBlock,
                                           (long long)ki.blocks_per_sm * E.sm_count);
    blocks = std::max<long long>(blocks, 1);
    double* d_out = (double*)ws.sums.ensure(sizeof(double) * (size_t)R * 4);
    void* args[] = {&k};
    if (trial) MCQ_CUDA(cudaEventRecord(trial->ev[variant][0], ws.stream));
    MCQ_CUDA(cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(kThreads), args, smem, ws.stream));
    if (trial) MCQ_CUDA(cudaEventRecord(trial->ev[variant][1], ws.stream));
    launch_finalize(k.partials, R, k.items_per_rep, 4, d_out, ws.stream);
    E.launches += 2;
    MCQ_CUDA(cudaGetLastError());
    std::vector<double> s((size_t)R * 4);
    MCQ_CUDA(cudaMemcpyAsync(s.data(), d_out, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, ws.stream));
    std::vector<double> nv(n_nodes);
    if (n_nodes)
        MCQ_CUDA(cudaMemcpyAsync(nv.data(), d_nodes, sizeof(double) * n_nodes, cudaMemcpyDeviceToHost, ws.stream));
    MCQ_CUDA(cudaStreamSynchronize(ws.stream));
    double mean[4] = {0, 0, 0, 0}, se[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; q++) {
        for (int r = 0; r < R; r++) mean[q] += s[4 * r + q] / (double)n_points;
        mean[q] /= R;
        double v = 0;
        for (int r = 0; r < R; r++) {
            const double d = s[4 * r + q] / (double)n_points - mean[q];
            v += d * d;
        }
        se[q] = R > 1 ? std::sqrt(v / (R - 1) / R) : 0.0;
    }
    out.price = mean[0]; out.delta = mean[1]; out.rho = mean[2]; out.vega = mean[3];
    out.price_se = se[0]; out.delta_se = se[1]; out.rho_se = se[2]; out.vega_se = se[3];
    out.n_paths = (int64_t)R * (int64_t)n_points;
    out.n_nodes = n_nodes;
    out.launches = E.launches - l0;
    out.path_steps = 3.0 * (double)out.n_paths * n_steps;   // forward + recompute + reverse
    if (node_vega)
        for (int i = 0; i < n_nodes; i++) node_vega[i] = nv[i] / (double)out.n_paths;
    out.time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace mcq
