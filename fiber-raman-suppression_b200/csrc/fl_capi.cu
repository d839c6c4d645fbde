// fl_capi.cu -- host runtime behind include/fiberlab_gpu.h: device tables,
// per-slot workspaces, kernel dispatch over the built grid sizes, and the
// C-ABI entry points.  Built for sm_100a only.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fiberlab_gpu.h"
#include "fl_launch.h"
#include "fl_mm_launch.h"

using namespace fl;

struct fl_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;  // the stream every call of this context runs on
    cudaStream_t own = nullptr;     // the context's private stream (the default for stream)
    std::string err;
    fl_ctx_opts opts{};
    long launches = 0;
    int sm_count = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // call start/end, kernel start/end
    double call_ms = 0.0, kernel_ms = 0.0;
};

namespace {

// NVTX range over a scope: the phases of a call (stepper launches,
// evaluation rounds, server launches, evidence) show up as named ranges in
// Nsight Systems and as ncu's --nvtx filter; without a tool attached a
// push/pop is a no-op call.
struct Nvtx {
    explicit Nvtx(const char* name) { nvtxRangePushA(name); }
    ~Nvtx() { nvtxRangePop(); }
    Nvtx(const Nvtx&) = delete;
    Nvtx& operator=(const Nvtx&) = delete;
};

int set_err(fl_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define CU(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? FL_ENOMEM : FL_ECUDA,  \
                           "%s failed: %s", #call, cudaGetErrorString(e_));              \
    } while (0)

int ilog2i(int n) {
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

bool pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

// physics_models.jl:438-449
bool hermitian(const double* hR, int nt) {
    double mx = 1.0;
    for (int k = 0; k < nt; k++) mx = std::max(mx, std::hypot(hR[2 * k], hR[2 * k + 1]));
    const double tol = 1e-12 * mx;
    if (std::fabs(hR[1]) > tol || std::fabs(hR[2 * (nt / 2) + 1]) > tol) return false;
    for (int k = 1; k < nt / 2; k++) {
        const int j = nt - k;
        const double ar = hR[2 * k], ai = hR[2 * k + 1], br = hR[2 * j], bi = -hR[2 * j + 1];
        const double d = std::hypot(ar - br, ai - bi);
        const double m = std::max(std::hypot(ar, ai), std::hypot(br, bi));
        if (d > std::max(tol, 1e-12 * m)) return false;
    }
    return true;
}

// sensitivity_disp_mmf.jl:103-112
bool gamma_symmetric(const double* g, int m) {
    double mx = 0.0;
    const long m4 = (long)m * m * m * m;
    for (long i = 0; i < m4; i++) mx = std::max(mx, std::fabs(g[i]));
    const double tol = 1e-12 * std::max(1.0, mx);
    auto at = [&](int i, int j, int k, int l) { return g[i + m * (j + m * (k + m * l))]; };
    auto close = [&](double a, double b) {
        return std::fabs(a - b) <= std::max(tol, 1e-12 * std::max(std::fabs(a), std::fabs(b)));
    };
    for (int l = 0; l < m; l++)
        for (int k = 0; k < m; k++)
            for (int j = 0; j < m; j++)
                for (int i = 0; i < m; i++) {
                    const double v = at(i, j, k, l);
                    if (!close(v, at(j, i, k, l)) || !close(v, at(i, k, j, l)) ||
                        !close(v, at(i, j, l, k)))
                        return false;
                }
    return true;
}

// u_shaped = u0 ⊙ cis(φ_b) (physics_models.jl:791-797): one phase per time
// bin shared by the modes, or (per_mode) one per (t, m)
__global__ void shaped_launch_kernel(const double2* __restrict__ u0,
                                     const double* __restrict__ phases, int nt, int m,
                                     int nbatch, double2* __restrict__ out, size_t out_stride,
                                     int per_mode = 0) {
    const long total = (long)nt * m * nbatch;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
         i += (long)gridDim.x * blockDim.x) {
        const int b = (int)(i / ((long)nt * m));
        const long q = i % ((long)nt * m);
        const int t = (int)(q % nt);
        double s, c;
        sincos(per_mode ? phases[(long)b * nt * m + q] : phases[(long)b * nt + t], &s, &c);
        const double2 x = u0[q];
        out[(size_t)b * out_stride + q] = make_double2(x.x * c - x.y * s, x.x * s + x.y * c);
    }
}

__global__ void gather_stats_kernel(const SlotState* __restrict__ st, int n,
                                    double* __restrict__ J) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) J[i] = st[i].J;
}

}  // namespace

struct fl_problem {
    fl_ctx* ctx = nullptr;
    int nt = 0, m = 0, precision = 0;
    double one_m_fR = 0, L = 0, reltol = 0, abstol = 0, gamma0 = 0;
    bool gamma_sym = true;
    int objective = OBJ_RAMAN_BAND;        // terminal objective of the gradient entry points
    double obj_tau = 50.0;                 // worst-mode smoothness
    bool use_mm = false;  // multimode runtime: M > 1, or M = 1 beyond one CTA's transform (2^15)
    double* d_Dturns = nullptr;
    void* d_Heff[2] = {nullptr, nullptr};  // [0] float, [1] double
    void* d_ss[2] = {nullptr, nullptr};
    void* d_tw[2] = {nullptr, nullptr};
    void* d_G[2] = {nullptr, nullptr};     // multimode contraction matrix [0] float, [1] double
    double* d_Ga = nullptr;                // its adjoint layout
    float* d_Gtc = nullptr;                // its tensor-core operand image (M >= 6)
    float* d_Gtcs = nullptr;               // its symmetric image (pairs i <= j; M >= 6)
    int rank = 0;                          // low-rank form of the contraction (0: not used)
    float* d_Vz = nullptr;                 // and its three tensor-core images
    float* d_Utc = nullptr;
    float* d_Utcs = nullptr;
    // device staging of the host-buffer batch calls (grow-only, reused)
    char* d_stage = nullptr;
    size_t stage_bytes = 0;
    // evidence reductions of the last forward's save positions (grow-only)
    double* d_ev = nullptr;
    size_t ev_bytes = 0;
    // workspace of the last forward (kept for fl_adjoint)
    struct Work* last = nullptr;
    struct MmWork* mlast = nullptr;        // same for multimode problems
};

// Per-batch workspace: one allocation carved into per-slot buffers.
struct Work {
    fl_ctx* ctx = nullptr;
    int B = 0, nt = 0, rsize = 4, K = 0, segcap = 0, stepcap = 0, nsave = 0;
    char* pool = nullptr;
    size_t pool_bytes = 0;
    void* d_desc = nullptr;          // SlotDesc[B]
    SlotState* d_state = nullptr;    // [B]
    int* d_active = nullptr;         // [B]
    std::vector<unsigned char> h_desc;  // host image of the descriptors
    double* d_u0 = nullptr;          // per-slot launch (B * nt complex)
    double* d_save = nullptr;        // per-slot save outputs (B * nsave * nt complex)
    double* d_lamL = nullptr;        // per-slot seed (B * nt complex)
    double* d_lam0 = nullptr;        // per-slot λ(0)
    double* d_grad = nullptr;        // per-slot gradient (B * nt)
    double* d_uL = nullptr;          // per-slot lab field at L
    double* d_zsave = nullptr;
    unsigned char* d_mask = nullptr;

    ~Work() {
        cudaFree(pool);
        cudaFree(d_desc);
        cudaFree(d_state);
        cudaFree(d_active);
    }
};

namespace {

// Accepted-step log entries per slot: the option, or (0) one per attempted
// step allowed, so the log never limits a solve that the attempted-step
// limit admits.
int step_log_entries(const fl_ctx_opts& o) {
    if (o.step_log > 0) return o.step_log;
    return (int)std::min<long>(o.max_iters, 1L << 30);
}

// rf: bytes of one forward-precision real (4 or 8); the adjoint is FP64
size_t slot_bytes(int nt, size_t rf, int K, int segcap, int stepcap) {
    const size_t C = 2 * rf * nt, D2 = 16 * (size_t)nt;
    size_t b = 0;
    b += 2 * D2 + 2 * D2;               // u[2], lam[2]
    b += 7 * C + 7 * D2;                // kf (RF), ka (FP64)
    b += 2 * D2 + D2 + 8 * (size_t)nt;  // scr[2], esv, skv
    b += (size_t)K * (D2 + C);          // checkpoints
    b += 16 * (size_t)stepcap;          // step log
    b += (size_t)segcap * 5 * C;        // recompute segment
    return b + 64 * 32;                 // alignment slack
}

char* carve(char*& p, size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~size_t(255);
    return r;
}

// Allocate a workspace for B slots; descriptors point into it.  Caller
// buffers (u0 etc.) are per-slot arrays inside the workspace.
int work_create(fl_problem* pr, int B, int nsave, int mode, Work** out,
                const fl_ctx_opts* opt = nullptr, cudaStream_t stream = nullptr) {
    const size_t rf = pr->precision == FL_PRECISION_FP64 ? 8 : 4;
    fl_ctx* ctx = pr->ctx;
    const fl_ctx_opts& o = opt ? *opt : ctx->opts;
    cudaStream_t strm = opt ? stream : ctx->stream;
    auto w = std::make_unique<Work>();
    w->ctx = ctx;
    w->B = B;
    w->nt = pr->nt;
    w->rsize = (int)rf;
    w->K = o.checkpoints;
    w->segcap = o.segment_steps;
    w->stepcap = step_log_entries(o);
    w->nsave = nsave;
    const int nt = pr->nt;
    const size_t per = slot_bytes(nt, rf, w->K, w->segcap, w->stepcap);
    const size_t io = 16 * (size_t)nt * (2 + nsave + 2) + 8 * (size_t)nt + 256 * 8;
    w->pool_bytes = (per + io) * (size_t)B + 16 * (size_t)std::max(nsave, 1) + nt + 4096;
    if (o.hbm_budget_bytes && w->pool_bytes > o.hbm_budget_bytes)
        return set_err(ctx, FL_OOM_ADMISSION, "workspace of %zu bytes exceeds the HBM budget",
                       w->pool_bytes);
    CU(cudaMalloc(&w->pool, w->pool_bytes));
    CU(cudaMalloc(&w->d_desc, sizeof(SlotDesc) * B));
    CU(cudaMalloc(&w->d_state, sizeof(SlotState) * B));
    CU(cudaMalloc(&w->d_active, sizeof(int) * B));
    char* p = w->pool;
    w->d_zsave = (double*)carve(p, 8 * (size_t)std::max(nsave, 1));
    w->d_mask = (unsigned char*)carve(p, nt);
    w->d_u0 = (double*)carve(p, 16 * (size_t)nt * B);
    w->d_lamL = (double*)carve(p, 16 * (size_t)nt * B);
    w->d_lam0 = (double*)carve(p, 16 * (size_t)nt * B);
    w->d_uL = (double*)carve(p, 16 * (size_t)nt * B);
    w->d_grad = (double*)carve(p, 8 * (size_t)nt * B);
    w->d_save = nsave ? (double*)carve(p, 16 * (size_t)nt * nsave * B) : nullptr;
    w->h_desc.resize(sizeof(SlotDesc) * B);
    SlotDesc* hd = reinterpret_cast<SlotDesc*>(w->h_desc.data());
    const size_t C = 2 * rf * nt, D2 = 16 * (size_t)nt;
    for (int b = 0; b < B; b++) {
        SlotDesc& d = hd[b];
        memset(&d, 0, sizeof d);
        d.Dturns = pr->d_Dturns;
        for (int q = 0; q < 2; q++) {
            d.Heff[q] = pr->d_Heff[q];
            d.ss[q] = pr->d_ss[q];
            d.tw[q] = pr->d_tw[q];
        }
        d.gamma = pr->gamma0;
        d.one_m_fR = pr->one_m_fR;
        d.L = pr->L;
        d.reltol = pr->reltol;
        d.abstol = pr->abstol;
        d.mode = mode;
        d.nsave = nsave;
        d.ck_cap = w->K;
        d.seg_cap = w->segcap;
        d.step_cap = w->stepcap;
        d.max_iters = o.max_iters;
        d.zsave = w->d_zsave;
        d.save_out = nsave ? w->d_save + (size_t)b * 2 * nt * nsave : nullptr;
        d.u0 = w->d_u0 + (size_t)b * 2 * nt;
        d.mask = w->d_mask;
        d.lamL = w->d_lamL + (size_t)b * 2 * nt;
        d.lam0_out = w->d_lam0 + (size_t)b * 2 * nt;
        d.grad_out = w->d_grad + (size_t)b * nt;
        d.uL_out = w->d_uL + (size_t)b * 2 * nt;
        d.u[0] = (double*)carve(p, D2);
        d.u[1] = (double*)carve(p, D2);
        d.lam[0] = (double*)carve(p, D2);
        d.lam[1] = (double*)carve(p, D2);
        for (int i = 0; i < 7; i++) d.kf[i] = carve(p, C);
        for (int i = 0; i < 7; i++) d.ka[i] = carve(p, D2);
        d.scr[0] = carve(p, D2);
        d.scr[1] = carve(p, D2);
        d.esv = (double*)carve(p, D2);
        d.skv = (double*)carve(p, 8 * (size_t)nt);
        d.ck_u = (double*)carve(p, D2 * w->K);
        d.ck_k1 = carve(p, C * w->K);
        d.steplog = (double*)carve(p, 16 * (size_t)w->stepcap);
        d.seg = carve(p, C * 5 * (size_t)w->segcap);
    }
    if ((size_t)(p - w->pool) > w->pool_bytes)
        return set_err(ctx, FL_ECUDA, "internal: workspace overflow (%zu > %zu)",
                       (size_t)(p - w->pool), w->pool_bytes);
    CU(cudaMemcpyAsync(w->d_desc, w->h_desc.data(), w->h_desc.size(), cudaMemcpyHostToDevice,
                       strm));
    std::vector<int> act(B);
    for (int b = 0; b < B; b++) act[b] = b;
    CU(cudaMemcpyAsync(w->d_active, act.data(), sizeof(int) * B, cudaMemcpyHostToDevice,
                       strm));
    CU(cudaMemsetAsync(w->d_state, 0, sizeof(SlotState) * B, strm));
    CU(cudaStreamSynchronize(strm));
    *out = w.release();
    return FL_OK;
}

int launch_slots(fl_ctx* ctx, fl_problem* pr, Work* w, int nactive, int max_evals) {
    const int logn = ilog2i(pr->nt);
    const int fp64 = pr->precision == FL_PRECISION_FP64;
    LaunchFn fn = sm_launcher(fp64, logn);
    if (!fn)
        return set_err(ctx, FL_EUNSUPPORTED, "Nt = 2^%d is not built for %s", logn,
                       fp64 ? "FP64" : "FP32");
    LaunchArgs a{w->d_desc, w->d_state, w->d_active, nactive, max_evals, ctx->stream};
    CU(fn(a));
    ctx->launches++;
    return FL_OK;
}

int run_to_completion(fl_problem* pr, Work* w) {
    Nvtx nvtx_("fl: single-mode stepper (run to completion)");
    fl_ctx* ctx = pr->ctx;
    CU(cudaEventRecord(ctx->ev[2], ctx->stream));
    int rc = launch_slots(ctx, pr, w, w->B, 0x7fffffff);
    if (rc) return rc;
    CU(cudaEventRecord(ctx->ev[3], ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
    ctx->kernel_ms = ms;
    return FL_OK;
}

int read_states(fl_ctx* ctx, Work* w, std::vector<SlotState>& st) {
    st.resize(w->B);
    CU(cudaMemcpyAsync(st.data(), w->d_state, sizeof(SlotState) * w->B, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

void fill_stats(const SlotState& s, fl_stats* o) {
    o->naccept = s.naccept;
    o->nreject = s.nreject;
    o->nf = s.nf;
    o->adj_naccept = s.a_naccept;
    o->adj_nreject = s.a_nreject;
    o->adj_nf = s.a_nf;
    o->status = s.status;
    o->checkpoints_used = s.ck_stride > 0 ? (s.nsteps + s.ck_stride - 1) / s.ck_stride : 0;
    o->J = s.J;
    o->z_end = s.z;
    o->recompute_steps = s.nrec;
}

int check_problem(fl_problem* pr) {
    if (!pr || !pr->ctx) return FL_EINVAL;
    return FL_OK;
}

template <typename R>
int upload_table_set(fl_problem* pr, const double* hR, const double* ss, int q) {
    fl_ctx* ctx = pr->ctx;
    const int nt = pr->nt;
    std::vector<R> heff(2 * (size_t)nt), ssv(nt), tw(2 * (size_t)nt);
    for (int k = 0; k < nt; k++) {
        const double sg = (k & 1) ? -1.0 : 1.0;  // fftshift folded into the response
        heff[2 * k] = (R)(hR[2 * k] * sg);
        heff[2 * k + 1] = (R)(hR[2 * k + 1] * sg);
        ssv[k] = (R)ss[k];
        const double a = -2.0 * M_PI * (double)k / (double)nt;
        tw[2 * k] = (R)std::cos(a);
        tw[2 * k + 1] = (R)std::sin(a);
    }
    CU(cudaMalloc(&pr->d_Heff[q], sizeof(R) * heff.size()));
    CU(cudaMalloc(&pr->d_ss[q], sizeof(R) * ssv.size()));
    CU(cudaMalloc(&pr->d_tw[q], sizeof(R) * tw.size()));
    CU(cudaMemcpy(pr->d_Heff[q], heff.data(), sizeof(R) * heff.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(pr->d_ss[q], ssv.data(), sizeof(R) * ssv.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(pr->d_tw[q], tw.data(), sizeof(R) * tw.size(), cudaMemcpyHostToDevice));
    return FL_OK;
}

// both precisions of the spectral tables (the adjoint is FP64 in every mode)
int upload_tables(fl_problem* pr, const double* D, const double* hR, const double* ss) {
    fl_ctx* ctx = pr->ctx;
    const int nt = pr->nt, m = pr->m;
    std::vector<double> dturn((size_t)nt * m);
    for (size_t i = 0; i < dturn.size(); i++) dturn[i] = D[i] / (2.0 * M_PI);
    CU(cudaMalloc(&pr->d_Dturns, sizeof(double) * dturn.size()));
    CU(cudaMemcpy(pr->d_Dturns, dturn.data(), sizeof(double) * dturn.size(),
                  cudaMemcpyHostToDevice));
    int rc = upload_table_set<float>(pr, hR, ss, 0);
    if (rc) return rc;
    return upload_table_set<double>(pr, hR, ss, 1);
}

int status_of_slots(fl_ctx* ctx, const std::vector<SlotState>& st) {
    for (size_t i = 0; i < st.size(); i++)
        if (st[i].status != ST_OK)
            return set_err(ctx, st[i].status, "slot %zu: %s", i, fl_status_string(st[i].status));
    return FL_OK;
}

int new_work(fl_problem* pr, int B, int nsave, int mode, Work** w) {
    return work_create(pr, B, nsave, mode, w);
}

// rewrite the mode (and the objective of a gradient mode) of every
// descriptor (host image + device copy)
int set_mode(fl_ctx* ctx, Work* w, int mode, int log_cost, int objective = OBJ_RAMAN_BAND,
             double tau = 50.0) {
    for (int b = 0; b < w->B; b++) {
        SlotDesc* d = reinterpret_cast<SlotDesc*>(w->h_desc.data()) + b;
        d->mode = mode;
        d->log_cost = log_cost;
        d->objective = objective;
        d->obj_tau = tau;
    }
    CU(cudaMemcpyAsync(w->d_desc, w->h_desc.data(), w->h_desc.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    return FL_OK;
}

// ---------------------------------------------------------------------------
// multimode (M > 1) runtime
// ---------------------------------------------------------------------------

}  // namespace

// Per-batch multimode workspace, carved like Work.
struct MmWork {
    fl_ctx* ctx = nullptr;
    int B = 0, nt = 0, m = 0, np = 0, K = 0, segcap = 0, stepcap = 0, nsave = 0;
    int per_mode = 0;
    char* pool = nullptr;
    size_t pool_bytes = 0;
    void* d_desc = nullptr;
    MmState* d_state = nullptr;
    int* d_active = nullptr;
    int* d_ndone = nullptr;
    int* h_ndone = nullptr;          // pinned
    std::vector<MmDesc> h_desc;
    double* d_u0 = nullptr;          // B * NM complex
    double* d_save = nullptr;        // B * nsave * NM complex
    double* d_lamL = nullptr;
    double* d_lam0 = nullptr;
    double* d_grad = nullptr;        // B * NM
    double* d_uL = nullptr;
    double* d_zsave = nullptr;
    unsigned char* d_mask = nullptr;
    // mm_run's batch of evaluation rounds as a CUDA graph, for graph_nactive slots
    cudaGraphExec_t graph = nullptr;
    int graph_nactive = -1;
    // the rounds' side stream and its fork / join events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    ~MmWork() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        cudaFree(pool);
        cudaFree(d_desc);
        cudaFree(d_state);
        cudaFree(d_active);
        cudaFree(d_ndone);
        cudaFreeHost(h_ndone);
    }
};

namespace {

size_t mm_slot_bytes(size_t nm, size_t npn, size_t rf, int K, int segcap, int stepcap, int nparts) {
    const size_t C = 2 * rf * nm, D2 = 16 * nm;
    size_t b = 0;
    b += 4 * D2;                         // u[2], lam[2]
    b += 7 * C + 7 * D2;                 // kf, ka
    b += 2 * D2 + 8 * nm + 8 * (size_t)nparts;  // probe, esv, skv, part
    b += (size_t)K * (D2 + C);           // checkpoints
    b += 16 * (size_t)stepcap;           // step log
    b += (size_t)segcap * 5 * C;         // recompute segment
    b += 3 * D2 + 2 * 8 * npn;           // ut, lt, eta, sq, cq
    return b + 40 * 256;                 // alignment of the carved buffers
}

int mm_work_create(fl_problem* pr, int B, int nsave, int mode, int per_mode, MmWork** out,
                   const fl_ctx_opts* opt = nullptr, cudaStream_t stream = nullptr) {
    fl_ctx* ctx = pr->ctx;
    const fl_ctx_opts& o = opt ? *opt : ctx->opts;
    cudaStream_t strm = opt ? stream : ctx->stream;
    const size_t rf = pr->precision == FL_PRECISION_FP64 ? 8 : 4;
    auto w = std::make_unique<MmWork>();
    w->ctx = ctx;
    w->B = B;
    w->nt = pr->nt;
    w->m = pr->m;
    w->np = pr->m * (pr->m + 1) / 2;
    w->K = o.checkpoints;
    w->segcap = o.segment_steps;
    w->stepcap = step_log_entries(o);
    w->nsave = nsave;
    w->per_mode = per_mode;
    const size_t nm = (size_t)pr->nt * pr->m, npn = (size_t)w->np * pr->nt;
    const int nparts = pr->m * mm_cluster_ctas(ilog2i(pr->nt));
    const size_t per = mm_slot_bytes(nm, npn, rf, w->K, w->segcap, w->stepcap, nparts);
    const size_t io = 16 * nm * (4 + nsave) + 8 * nm + 256 * 8;
    w->pool_bytes = (per + io) * (size_t)B + 16 * (size_t)std::max(nsave, 1) + pr->nt + 4096;
    if (o.hbm_budget_bytes && w->pool_bytes > o.hbm_budget_bytes)
        return set_err(ctx, FL_OOM_ADMISSION, "workspace of %zu bytes exceeds the HBM budget",
                       w->pool_bytes);
    CU(cudaMalloc(&w->pool, w->pool_bytes));
    CU(cudaMalloc(&w->d_desc, sizeof(MmDesc) * B));
    CU(cudaMalloc(&w->d_state, sizeof(MmState) * B));
    CU(cudaStreamCreateWithFlags(&w->side, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&w->ev_fork, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&w->ev_join, cudaEventDisableTiming));
    CU(cudaMalloc(&w->d_active, sizeof(int) * B));
    CU(cudaMalloc(&w->d_ndone, sizeof(int)));
    CU(cudaMallocHost(&w->h_ndone, sizeof(int)));
    char* p = w->pool;
    w->d_zsave = (double*)carve(p, 8 * (size_t)std::max(nsave, 1));
    w->d_mask = (unsigned char*)carve(p, pr->nt);
    w->d_u0 = (double*)carve(p, 16 * nm * B);
    w->d_lamL = (double*)carve(p, 16 * nm * B);
    w->d_lam0 = (double*)carve(p, 16 * nm * B);
    w->d_uL = (double*)carve(p, 16 * nm * B);
    w->d_grad = (double*)carve(p, 8 * nm * B);
    w->d_save = nsave ? (double*)carve(p, 16 * nm * nsave * B) : nullptr;
    w->h_desc.assign(B, MmDesc{});
    const size_t C = 2 * rf * nm, D2 = 16 * nm;
    for (int b = 0; b < B; b++) {
        MmDesc& d = w->h_desc[b];
        d.Dturns = pr->d_Dturns;
        for (int q = 0; q < 2; q++) {
            d.Heff[q] = pr->d_Heff[q];
            d.ss[q] = pr->d_ss[q];
            d.tw[q] = pr->d_tw[q];
            d.G[q] = pr->d_G[q];
        }
        d.Ga = pr->d_Ga;
        d.Gtc = pr->d_Gtc;
        d.Gtcs = pr->d_Gtcs;
        d.rank = pr->rank;
        d.Vz = pr->d_Vz;
        d.Utc = pr->d_Utc;
        d.Utcs = pr->d_Utcs;
        d.M = pr->m;
        d.nparts = nparts;
        d.NP = w->np;
        d.N = pr->nt;
        d.fp64 = pr->precision == FL_PRECISION_FP64;
        d.adj_mixed = mm_adj_mixed(d.M, d.N, d.fp64);
        d.one_m_fR = pr->one_m_fR;
        d.L = pr->L;
        d.reltol = pr->reltol;
        d.abstol = pr->abstol;
        d.mode = mode;
        d.log_cost = 0;
        d.nsave = nsave;
        d.phase_per_mode = per_mode;
        d.ck_cap = w->K;
        d.seg_cap = w->segcap;
        d.step_cap = w->stepcap;
        d.max_iters = o.max_iters;
        d.zsave = w->d_zsave;
        d.save_out = nsave ? w->d_save + (size_t)b * 2 * nm * nsave : nullptr;
        d.u0 = w->d_u0 + (size_t)b * 2 * nm;
        d.mask = w->d_mask;
        d.lamL = w->d_lamL + (size_t)b * 2 * nm;
        d.lam0_out = w->d_lam0 + (size_t)b * 2 * nm;
        d.grad_out = w->d_grad + (size_t)b * nm;
        d.uL_out = w->d_uL + (size_t)b * 2 * nm;
        for (int i = 0; i < 2; i++) d.u[i] = (double*)carve(p, D2);
        for (int i = 0; i < 2; i++) d.lam[i] = (double*)carve(p, D2);
        for (int i = 0; i < 7; i++) d.kf[i] = carve(p, C);
        for (int i = 0; i < 7; i++) d.ka[i] = carve(p, D2);
        d.probe = carve(p, D2);
        d.esv = (double*)carve(p, D2);
        d.skv = (double*)carve(p, 8 * nm);
        d.part = (double*)carve(p, 8 * (size_t)nparts);
        d.ck_u = (double*)carve(p, D2 * w->K);
        d.ck_k1 = carve(p, C * w->K);
        d.steplog = (double*)carve(p, 16 * (size_t)w->stepcap);
        d.seg = carve(p, C * 5 * (size_t)w->segcap);
        d.ut = carve(p, D2);
        d.lt = carve(p, D2);
        d.eta = carve(p, D2);
        d.sq = carve(p, 8 * npn);
        d.cq = carve(p, 8 * npn);
    }
    if ((size_t)(p - w->pool) > w->pool_bytes)
        return set_err(ctx, FL_ECUDA, "internal: workspace overflow (%zu > %zu)",
                       (size_t)(p - w->pool), w->pool_bytes);
    CU(cudaMemcpyAsync(w->d_desc, w->h_desc.data(), sizeof(MmDesc) * B, cudaMemcpyHostToDevice,
                       strm));
    std::vector<int> act(B);
    for (int b = 0; b < B; b++) act[b] = b;
    CU(cudaMemcpyAsync(w->d_active, act.data(), sizeof(int) * B, cudaMemcpyHostToDevice,
                       strm));
    CU(cudaMemsetAsync(w->d_state, 0, sizeof(MmState) * B, strm));
    CU(cudaStreamSynchronize(strm));
    *out = w.release();
    return FL_OK;
}

int mm_set_mode(fl_ctx* ctx, MmWork* w, int mode, int log_cost, int objective = OBJ_RAMAN_BAND,
                double tau = 50.0) {
    for (auto& d : w->h_desc) {
        d.mode = mode;
        d.log_cost = log_cost;
        d.objective = objective;
        d.obj_tau = tau;
    }
    CU(cudaMemcpyAsync(w->d_desc, w->h_desc.data(), sizeof(MmDesc) * w->B, cudaMemcpyHostToDevice,
                       ctx->stream));
    return FL_OK;
}

MmRound mm_round_args(fl_problem* pr, MmWork* w, int nactive) {
    MmRound a{};
    a.desc = w->d_desc;
    a.state = w->d_state;
    a.active = w->d_active;
    a.nactive = nactive;
    a.M = pr->m;
    a.NP = w->np;
    a.N = pr->nt;
    a.fp64 = pr->precision == FL_PRECISION_FP64;
    a.lowrank_some = pr->rank > 0;  // one problem per batch
    a.fullrank_some = pr->rank == 0;
    a.side = w->side;
    a.ev_fork = w->ev_fork;
    a.ev_join = w->ev_join;
    a.control = 1;
    a.tensor_cores = 1;
    a.ndone = nullptr;
    a.stream = pr->ctx->stream;
    return a;
}

// Evaluation rounds until every one of the first nactive slots is done: one
// control pass prepares each slot's first evaluation, then batches of rounds
// run with the finished-slot count read back after each batch.  Every slot
// has its own attempted-step limits, so the loop ends; the host bound below
// only guards against a control bug.
int mm_run(fl_problem* pr, MmWork* w, int nactive) {
    Nvtx nvtx_("fl: multimode evaluation rounds");
    fl_ctx* ctx = pr->ctx;
    MmRoundFn round = mm_round_launcher(ilog2i(pr->nt));
    if (!round) return set_err(ctx, FL_EUNSUPPORTED, "multimode Nt = %d is not built", pr->nt);
    MmRound a = mm_round_args(pr, w, nactive);
    CU(cudaEventRecord(ctx->ev[2], ctx->stream));
    CU(mm_launch_control(a, 0));
    ctx->launches++;
    const int per_batch = 8;
    // one batch: 8 evaluation rounds, the counter of finished slots reset
    // before the last round (which counts them)
    auto enqueue_batch = [&](cudaStream_t cs) -> cudaError_t {
        MmRound b = a;
        b.stream = cs;
        for (int r = 0; r < per_batch; r++) {
            b.ndone = nullptr;
            if (r == per_batch - 1) {
                const cudaError_t e = cudaMemsetAsync(w->d_ndone, 0, sizeof(int), cs);
                if (e != cudaSuccess) return e;
                b.ndone = w->d_ndone;
            }
            const cudaError_t e = round(b);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    // The batch is captured once as a CUDA graph and replayed: each kernel
    // reads every slot's phase from device memory, so the same launches serve
    // every batch, and a batch costs one graph launch instead of 8 x 7..10
    // kernel launches.  Capture is thread-local (other host threads, e.g. a
    // server's, keep launching) and runs on the context's private stream, so
    // a caller's stream (which may be the legacy default stream) is never put
    // in capture mode; the graph is launched on the context's current stream.
    if (!w->graph || w->graph_nactive != nactive) {
        if (w->graph) cudaGraphExecDestroy(w->graph);
        w->graph = nullptr;
        w->graph_nactive = -1;
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(ctx->own, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e1 = enqueue_batch(ctx->own);
        const cudaError_t e2 = cudaStreamEndCapture(ctx->own, &g);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return set_err(ctx, FL_ECUDA, "capturing the evaluation batch: %s",
                           cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        }
        const cudaError_t e3 = cudaGraphInstantiate(&w->graph, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            w->graph = nullptr;
            return set_err(ctx, FL_ECUDA, "instantiating the evaluation batch: %s",
                           cudaGetErrorString(e3));
        }
        w->graph_nactive = nactive;
    }
    const long max_rounds = 4 * 7 * (ctx->opts.max_iters + 2) + 64;
    long rounds = 0;
    for (;;) {
        CU(cudaGraphLaunch(w->graph, ctx->stream));
        ctx->launches += per_batch * (a.fp64 ? 7 : 10);
        rounds += per_batch;
        CU(cudaMemcpyAsync(w->h_ndone, w->d_ndone, sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        if (*w->h_ndone >= nactive) break;
        if (rounds > max_rounds)
            return set_err(ctx, FL_MAXITERS, "multimode stepper did not finish in %ld rounds",
                           rounds);
    }
    CU(cudaEventRecord(ctx->ev[3], ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
    ctx->kernel_ms = ms;
    return FL_OK;
}

int mm_read_states(fl_ctx* ctx, MmWork* w, int n, std::vector<MmState>& st) {
    st.resize(n);
    CU(cudaMemcpyAsync(st.data(), w->d_state, sizeof(MmState) * n, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

void mm_fill_stats(const MmState& s, fl_stats* o) {
    o->naccept = s.naccept;
    o->nreject = s.nreject;
    o->nf = s.nf;
    o->adj_naccept = s.a_naccept;
    o->adj_nreject = s.a_nreject;
    o->adj_nf = s.a_nf;
    o->status = s.status;
    o->checkpoints_used = s.ck_stride > 0 ? (s.nsteps + s.ck_stride - 1) / s.ck_stride : 0;
    o->J = s.J;
    o->z_end = s.z;
    o->recompute_steps = s.nrec;
}

__global__ void mm_gather_J_kernel(const MmState* __restrict__ st, int n, double* __restrict__ J) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) J[i] = st[i].J;
}

// G[(i*M + j)*GP + q] = γ[i,j,k,l] + γ[i,j,l,k] (k < l), γ[i,j,k,k] (k = l),
// q enumerating k <= l row by row (GP: the pair count padded to 4 with zeros);
// the adjoint's copy Ga[(j*NP + q)*MP + i] (MP: M padded to 2); γ in the
// reference's column-major order
// Eigen-decomposition of a symmetric n x n matrix (row-major; destroyed) by
// cyclic Jacobi rotations: eigenvalues in w, eigenvectors as the columns of v.
void sym_eig(std::vector<double>& a, int n, std::vector<double>& w, std::vector<double>& v) {
    v.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) v[(size_t)i * n + i] = 1.0;
    double tot = 0.0;
    for (double x : a) tot += x * x;
    for (int sweep = 0; sweep < 64; sweep++) {
        double off = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) off += a[(size_t)p * n + q] * a[(size_t)p * n + q];
        if (off <= 1e-32 * tot) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = a[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double th = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2.0 * apq);
                const double t = (th >= 0.0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < n; k++) {  // columns p, q
                    const double x = a[(size_t)k * n + p], y = a[(size_t)k * n + q];
                    a[(size_t)k * n + p] = c * x - sn * y;
                    a[(size_t)k * n + q] = sn * x + c * y;
                }
                for (int k = 0; k < n; k++) {  // rows p, q
                    const double x = a[(size_t)p * n + k], y = a[(size_t)q * n + k];
                    a[(size_t)p * n + k] = c * x - sn * y;
                    a[(size_t)q * n + k] = sn * x + c * y;
                }
                for (int k = 0; k < n; k++) {
                    const double x = v[(size_t)k * n + p], y = v[(size_t)k * n + q];
                    v[(size_t)k * n + p] = c * x - sn * y;
                    v[(size_t)k * n + q] = sn * x + c * y;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; i++) w[i] = a[(size_t)i * n + i];
}

// TF32 round to nearest of an FP32 value (10-bit mantissa; the tensor cores'
// operand format), the host side of the 3xTF32 split
float tf32_host(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

// A tensor-core B operand image: rows x K (K a multiple of 8, rows a multiple
// of 8) in the K-major no-swizzle shared-memory layout, split hi then lo.
template <class F>
std::vector<unsigned char> tc_image(int rows, int K, F&& f) {
    const size_t bytes = (size_t)rows * K * 4;
    std::vector<unsigned char> img(2 * bytes, 0);
    for (int r = 0; r < rows; r++)
        for (int k = 0; k < K; k++) {
            const float g = f(r, k);
            if (g == 0.f) continue;
            const float hi = tf32_host(g), lo = tf32_host(g - hi);
            const uint32_t off = (uint32_t)((r >> 3) * (K * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
            memcpy(&img[off], &hi, 4);
            memcpy(&img[bytes + off], &lo, 4);
        }
    return img;
}

int upload_image(fl_ctx* ctx, const std::vector<unsigned char>& img, float** dst) {
    CU(cudaMalloc(dst, img.size()));
    CU(cudaMemcpy(*dst, img.data(), img.size(), cudaMemcpyHostToDevice));
    return FL_OK;
}

// The low-rank form of the pair contraction (symmetric γ, FP32 batches with
// M >= 6): the Gram matrix Γ[p][q] = γ_ijkl of the pairs p = (i <= j),
// q = (k <= l) has rank dim span{φ_i φ_j}, often well below NP (28 of 55 for
// the ten Hermite-Gauss modes with m + n <= 3, whose products are a Gaussian
// times the 28 monomials of degree <= 6).  With Γ = Σ_k λ_k Q_k Q_kᵀ over the
// eigenvalues above 1e-12 of the largest and G[ij][q] = w_q Γ[p][q] (w_q = 2
// for k < l), every contraction with G factors as
//   Σ_q G[ij][q] X_q = Σ_k U[p][k] Z_k,  U[p][k] = λ_k Q[p][k],
//   Z_k = Σ_q V[q][k] X_q,  V[q][k] = w_q Q[q][k],
// and the FP32 path convolves the r sequences Z_k instead of the NP pair
// products.  Used when it saves at least one pair transform.
int mm_lowrank_setup(fl_problem* pr, const double* gamma) {
    const int M = pr->m, NP = M * (M + 1) / 2, KP = (NP + 7) & ~7;
    auto g = [&](int i, int j, int k, int l) { return gamma[i + M * (j + M * (k + M * l))]; };
    std::vector<int> pk(NP), pl(NP);
    for (int k = 0, q = 0; k < M; k++)
        for (int l = k; l < M; l++, q++) {
            pk[q] = k;
            pl[q] = l;
        }
    std::vector<double> Gam((size_t)NP * NP), lam, Q;
    for (int p = 0; p < NP; p++)
        for (int q = 0; q < NP; q++) Gam[(size_t)p * NP + q] = g(pk[p], pl[p], pk[q], pl[q]);
    sym_eig(Gam, NP, lam, Q);
    std::vector<int> ord(NP);
    for (int i = 0; i < NP; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return std::fabs(lam[a]) > std::fabs(lam[b]); });
    const double lmax = std::fabs(lam[ord[0]]);
    int r = 0;
    while (r < NP && std::fabs(lam[ord[r]]) > 1e-12 * lmax) r++;
    // used when it saves pair transforms and the rank fits the kernels' tables
    if (r == 0 || (r + 1) / 2 >= (NP + 1) / 2 || ((r + 7) & ~7) > mm_krmax(M)) return FL_OK;
    const int KR = (r + 7) & ~7, NZ = (r + 15) & ~15, NN = (M * M + 15) & ~15, NS = (NP + 15) & ~15;
    auto U = [&](int p, int k) { return k < r ? (float)(lam[ord[k]] * Q[(size_t)p * NP + ord[k]]) : 0.f; };
    auto pidx = [&](int i, int j) {
        const int a = std::min(i, j), b = std::max(i, j);
        return a * M - a * (a - 1) / 2 + (b - a);
    };
    int rc = upload_image(pr->ctx, tc_image(NZ, KP, [&](int k, int q) {
        return k < r && q < NP ? (float)((pk[q] == pl[q] ? 1.0 : 2.0) * Q[(size_t)q * NP + ord[k]]) : 0.f;
    }), &pr->d_Vz);
    if (!rc) rc = upload_image(pr->ctx, tc_image(NN, KR, [&](int row, int k) {
        return row < M * M ? U(pidx(row / M, row % M), k) : 0.f;
    }), &pr->d_Utc);
    if (!rc) rc = upload_image(pr->ctx, tc_image(NS, KR, [&](int p, int k) { return p < NP ? U(p, k) : 0.f; }),
                               &pr->d_Utcs);
    if (rc) return rc;
    pr->rank = r;
    return FL_OK;
}

int mm_upload_G(fl_problem* pr, const double* gamma) {
    fl_ctx* ctx = pr->ctx;
    const int M = pr->m, NP = M * (M + 1) / 2, GP = mm_gp(M), MP = mm_mp(M);
    auto g = [&](int i, int j, int k, int l) { return gamma[i + M * (j + M * (k + M * l))]; };
    std::vector<double> G((size_t)M * M * GP, 0.0), Ga((size_t)M * NP * MP, 0.0);
    std::vector<float> Gf(G.size(), 0.f);
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) {
            int q = 0;
            for (int k = 0; k < M; k++)
                for (int l = k; l < M; l++, q++) {
                    const double v = k == l ? g(i, j, k, k) : g(i, j, k, l) + g(i, j, l, k);
                    G[((size_t)i * M + j) * GP + q] = v;
                    Gf[((size_t)i * M + j) * GP + q] = (float)v;
                    Ga[((size_t)j * NP + q) * MP + i] = v;
                }
        }
    CU(cudaMalloc(&pr->d_G[0], sizeof(float) * Gf.size()));
    CU(cudaMalloc(&pr->d_G[1], sizeof(double) * G.size()));
    CU(cudaMalloc(&pr->d_Ga, sizeof(double) * Ga.size()));
    CU(cudaMemcpy(pr->d_G[0], Gf.data(), sizeof(float) * Gf.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(pr->d_G[1], G.data(), sizeof(double) * G.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(pr->d_Ga, Ga.data(), sizeof(double) * Ga.size(), cudaMemcpyHostToDevice));
    if (M >= 6) {
        // B operand of the tensor-core contraction: rows ij (padded to a multiple
        // of 16), pairs (padded to 8), split into TF32 hi + lo (round to
        // nearest: 10-bit mantissa), laid out as the kernel's shared memory
        const int KP = (NP + 7) & ~7, NN = (M * M + 15) & ~15;
        const size_t bbytes = (size_t)NN * KP * 4;
        std::vector<unsigned char> img(2 * bbytes, 0);
        auto tf32 = [](float x) {
            uint32_t u;
            memcpy(&u, &x, 4);
            if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
            float r;
            memcpy(&r, &u, 4);
            return r;
        };
        for (int r = 0; r < M * M; r++)
            for (int k = 0; k < NP; k++) {
                const float g = Gf[(size_t)r * GP + k];
                const float hi = tf32(g), lo = tf32(g - hi);
                const uint32_t off = (uint32_t)((r >> 3) * (KP * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
                memcpy(&img[off], &hi, 4);
                memcpy(&img[bbytes + off], &lo, 4);
            }
        CU(cudaMalloc(&pr->d_Gtc, img.size()));
        CU(cudaMemcpy(pr->d_Gtc, img.data(), img.size(), cudaMemcpyHostToDevice));
        // the symmetric B operand of the adjoint contractions: row p holds
        // G[i][j][.] = G[j][i][.] for the pairs p = (i <= j) (rows padded to
        // 16 with zeros), the same pairs along K, split and layout
        const int NS = (NP + 15) & ~15;
        const size_t abytes = (size_t)NS * KP * 4;
        std::vector<unsigned char> aimg(2 * abytes, 0);
        for (int i = 0, r = 0; i < M; i++)
            for (int j = i; j < M; j++, r++)
                for (int k = 0; k < NP; k++) {
                    const float g = Gf[((size_t)i * M + j) * GP + k];
                    const float hi = tf32(g), lo = tf32(g - hi);
                    const uint32_t off =
                        (uint32_t)((r >> 3) * (KP * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
                    memcpy(&aimg[off], &hi, 4);
                    memcpy(&aimg[abytes + off], &lo, 4);
                }
        CU(cudaMalloc(&pr->d_Gtcs, aimg.size()));
        CU(cudaMemcpy(pr->d_Gtcs, aimg.data(), aimg.size(), cudaMemcpyHostToDevice));
        if (pr->gamma_sym && mm_adj_mixed(M, pr->nt, pr->precision == FL_PRECISION_FP64)) {
            const int rc = mm_lowrank_setup(pr, gamma);
            if (rc) return rc;
        }
    }
    return FL_OK;
}

int mm_forward(fl_problem* pr, const double* u0, const double* saveat, int nsave,
               double* out_spectra, fl_stats* stats) {
    fl_ctx* ctx = pr->ctx;
    const size_t nm = (size_t)pr->nt * pr->m;
    // the problem's one-slot forward workspace is reused by later forwards
    // with the same number of save positions (no allocation per call)
    MmWork* w = pr->mlast;
    int rc = FL_OK;
    if (w && w->B == 1 && w->nsave == nsave && !w->per_mode) {
        rc = mm_set_mode(ctx, w, MODE_FORWARD, 0);
        if (rc) return rc;
        CU(cudaMemsetAsync(w->d_state, 0, sizeof(MmState), ctx->stream));
    } else {
        delete pr->mlast;
        pr->mlast = nullptr;
        w = nullptr;
        rc = mm_work_create(pr, 1, nsave, MODE_FORWARD, 0, &w);
        if (rc) return rc;
        pr->mlast = w;
    }
    CU(cudaMemcpyAsync(w->d_u0, u0, 16 * nm, cudaMemcpyHostToDevice, ctx->stream));
    if (nsave)
        CU(cudaMemcpyAsync(w->d_zsave, saveat, 8 * (size_t)nsave, cudaMemcpyHostToDevice,
                           ctx->stream));
    rc = mm_run(pr, w, 1);
    if (rc) return rc;
    std::vector<MmState> st;
    rc = mm_read_states(ctx, w, 1, st);
    if (rc) return rc;
    if (stats) mm_fill_stats(st[0], stats);
    if (st[0].status) return set_err(ctx, st[0].status, "%s", fl_status_string(st[0].status));
    if (nsave) CU(cudaMemcpy(out_spectra, w->d_save, 16 * nm * nsave, cudaMemcpyDeviceToHost));
    return FL_OK;
}

int mm_adjoint(fl_problem* pr, const double* lambdaL, double* lambda0, fl_stats* stats) {
    fl_ctx* ctx = pr->ctx;
    const size_t nm = (size_t)pr->nt * pr->m;
    MmWork* w = pr->mlast;
    std::vector<MmState> st;
    int rc = mm_read_states(ctx, w, 1, st);
    if (rc) return rc;
    if (st[0].phase != PH_DONE || st[0].status != ST_OK)
        return set_err(ctx, FL_EINVAL, "the last forward did not complete");
    st[0].phase = PH_SEED;
    CU(cudaMemcpyAsync(w->d_state, st.data(), sizeof(MmState), cudaMemcpyHostToDevice,
                       ctx->stream));
    rc = mm_set_mode(ctx, w, MODE_SEEDED_ADJOINT, 0);
    if (rc) return rc;
    CU(cudaMemcpyAsync(w->d_lamL, lambdaL, 16 * nm, cudaMemcpyHostToDevice, ctx->stream));
    rc = mm_run(pr, w, 1);
    if (rc) return rc;
    rc = mm_read_states(ctx, w, 1, st);
    if (rc) return rc;
    if (stats) mm_fill_stats(st[0], stats);
    if (st[0].status) return set_err(ctx, st[0].status, "%s", fl_status_string(st[0].status));
    CU(cudaMemcpy(lambda0, w->d_lam0, 16 * nm, cudaMemcpyDeviceToHost));
    return FL_OK;
}

// one RHS evaluation through the multimode kernels (no control pass)
int mm_rhs_eval(fl_problem* pr, int adjoint, double z, const double* u_in, const double* u_fwd,
                double* du_out) {
    fl_ctx* ctx = pr->ctx;
    const size_t nm = (size_t)pr->nt * pr->m;
    MmRoundFn round = mm_round_launcher(ilog2i(pr->nt));
    if (!round) return set_err(ctx, FL_EUNSUPPORTED, "multimode Nt = %d is not built", pr->nt);
    MmWork* w = nullptr;
    int rc = mm_work_create(pr, 1, 0, MODE_FORWARD, 0, &w);
    if (rc) return rc;
    std::unique_ptr<MmWork> hold(w);
    CU(cudaMemcpyAsync(w->d_u0, u_in, 16 * nm, cudaMemcpyHostToDevice, ctx->stream));
    if (adjoint) CU(cudaMemcpyAsync(w->d_lamL, u_fwd, 16 * nm, cudaMemcpyHostToDevice, ctx->stream));
    MmState st{};
    st.phase = adjoint ? PH_EVAL_ADJ : PH_EVAL_FWD;
    st.ez = st.ezload = z;
    CU(cudaMemcpyAsync(w->d_state, &st, sizeof st, cudaMemcpyHostToDevice, ctx->stream));
    MmRound a = mm_round_args(pr, w, 1);
    a.control = 0;
    CU(round(a));
    ctx->launches += a.fp64 ? 6 : 9;
    CU(cudaMemcpyAsync(du_out, w->d_lam0, 16 * nm, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

// batched forward + band objective + adjoint + phase gradient of the
// multimode stepper on device buffers; phases (Nt, B) shared by the modes or
// (Nt, M, B) per mode; grad has the shape of the phases
int mm_phase_gradient_device(fl_problem* pr, const double* d_u0, int nbatch,
                             const double* d_phases, int per_mode, const unsigned char* d_mask,
                             int log_cost, double* d_J, double* d_grad, fl_stats* stats) {
    Nvtx nvtx_("fl: multimode batched forward + adjoint + gradient");
    fl_ctx* ctx = pr->ctx;
    const int nt = pr->nt;
    const size_t nm = (size_t)nt * pr->m;
    if (!pr->mlast || pr->mlast->B < nbatch || pr->mlast->nsave != 0 ||
        pr->mlast->per_mode != per_mode) {
        delete pr->mlast;
        pr->mlast = nullptr;
        MmWork* w = nullptr;
        int rc = mm_work_create(pr, nbatch, 0, MODE_BAND_GRADIENT, per_mode, &w);
        if (rc) return rc;
        pr->mlast = w;
    }
    MmWork* w = pr->mlast;
    CU(cudaEventRecord(ctx->ev[0], ctx->stream));
    int rc = mm_set_mode(ctx, w, MODE_BAND_GRADIENT, log_cost, pr->objective, pr->obj_tau);
    if (rc) return rc;
    CU(cudaMemsetAsync(w->d_state, 0, sizeof(MmState) * nbatch, ctx->stream));
    CU(cudaMemcpyAsync(w->d_mask, d_mask, nt, cudaMemcpyDeviceToDevice, ctx->stream));
    const int threads = 256;
    const long total = (long)nm * nbatch;
    const int blocks = (int)std::min<long>((total + threads - 1) / threads, 4096);
    shaped_launch_kernel<<<blocks, threads, 0, ctx->stream>>>(
        (const double2*)d_u0, d_phases, nt, pr->m, nbatch, (double2*)w->d_u0, nm, per_mode);
    ctx->launches++;
    CU(cudaGetLastError());
    rc = mm_run(pr, w, nbatch);
    if (rc) return rc;
    mm_gather_J_kernel<<<(nbatch + 255) / 256, 256, 0, ctx->stream>>>(w->d_state, nbatch, d_J);
    ctx->launches++;
    CU(cudaGetLastError());
    // per-slot gradients are NM apart; the caller's are N (shared) or NM (per mode) apart
    const size_t gl = per_mode ? nm : (size_t)nt;
    CU(cudaMemcpy2DAsync(d_grad, 8 * gl, w->d_grad, 8 * nm, 8 * gl, nbatch,
                         cudaMemcpyDeviceToDevice, ctx->stream));
    CU(cudaEventRecord(ctx->ev[1], ctx->stream));
    std::vector<MmState> st;
    rc = mm_read_states(ctx, w, nbatch, st);
    if (rc) return rc;
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->call_ms = ms;
    if (stats)
        for (int b = 0; b < nbatch; b++) mm_fill_stats(st[b], &stats[b]);
    for (int b = 0; b < nbatch; b++)
        if (st[b].status != ST_OK)
            return set_err(ctx, st[b].status, "slot %d: %s", b, fl_status_string(st[b].status));
    return FL_OK;
}

// ---------------------------------------------------------------------------
// serving runtime
// ---------------------------------------------------------------------------

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

}  // namespace

struct SrvRequest {
    long id = 0;
    int weight = 1;                    // CTAs per transform of its slot
    fl_problem* prob = nullptr;
    int kind = FL_REQ_FORWARD, log_cost = 0;
    int objective = OBJ_RAMAN_BAND;    // the problem's objective when submitted
    double obj_tau = 50.0;
    double L = 0;
    std::vector<double> u0;            // shaped launch, (Nt, M) complex
    std::vector<unsigned char> mask;
    double* out_field = nullptr;
    double* out_grad = nullptr;
    int status = FL_EBUSY;
    fl_stats stats{};
    double J = 0, t_submit = 0, t_done = 0;
};

// One chunk of slots of one bucket, advanced on its own stream.
struct SrvChunk {
    bool mm = false;
    Work* w = nullptr;
    MmWork* mw = nullptr;
    int B = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    bool inflight = false;
    std::vector<SrvRequest*> slot;     // nullptr: free
    unsigned char* d_masks = nullptr;  // per-slot band masks (B * Nt)
    size_t bytes = 0;
    std::vector<SlotState> hs;
    std::vector<MmState> hms;
    cudaGraphExec_t graph = nullptr;   // multimode: one launch's rounds, captured once
    ~SrvChunk() {
        if (graph) cudaGraphExecDestroy(graph);
        delete w;
        delete mw;
        cudaFree(d_masks);
        if (ev) cudaEventDestroy(ev);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Requests of one shape (Nt, M, precision): slots of one chunk share the
// kernel instance; each slot's descriptor points at its request's tables.
struct SrvBucket {
    int nt = 0, m = 0, precision = 0;
    bool mm = false;
    fl_problem* tables = nullptr;      // server-owned twiddles (and defaults) for free slots
    std::vector<SrvChunk*> chunks;
    ~SrvBucket() {
        for (auto* c : chunks) delete c;
        if (tables) fl_problem_destroy(tables);
    }
};

struct fl_server {
    fl_ctx* ctx = nullptr;
    fl_server_opts opts{};
    fl_ctx_opts wopts{};
    std::mutex mu;
    std::condition_variable cv;
    std::map<long, SrvRequest*> reqs;
    std::deque<SrvRequest*> incoming;      // submitted, not yet seen by the progress thread
    std::deque<SrvRequest*> waiting;       // arrival order, not yet in a slot (progress thread)
    std::atomic<long> n_waiting{0};
    long active_w = 0;                     // CTAs per transform of the requests in slots
    std::vector<SrvBucket*> buckets;
    size_t hbm_used = 0;
    long next_id = 1, submitted = 0, completed = 0, launches = 0;
    int fatal = FL_OK;
    std::string err;
    std::atomic<bool> stop{false};
    std::thread th;
};

namespace {

// slot footprint of one request of this shape, with the server's options
size_t srv_slot_bytes(const fl_server* sv, const fl_problem* pr) {
    const size_t rf = pr->precision == FL_PRECISION_FP64 ? 8 : 4;
    const fl_ctx_opts& o = sv->wopts;
    if (!pr->use_mm) return slot_bytes(pr->nt, rf, o.checkpoints, o.segment_steps,
                                       step_log_entries(o)) +
                            16 * (size_t)pr->nt * 4 + 8 * (size_t)pr->nt + 2 * (size_t)pr->nt;
    const size_t nm = (size_t)pr->nt * pr->m, np = (size_t)pr->m * (pr->m + 1) / 2;
    return mm_slot_bytes(nm, np * pr->nt, rf, o.checkpoints, o.segment_steps, step_log_entries(o),
                         pr->m * mm_cluster_ctas(ilog2i(pr->nt))) +
           16 * nm * 4 + 8 * nm + 2 * (size_t)pr->nt;
}

int srv_chunk_slots(const fl_server* sv, const SrvBucket* b) {
    const int cap = std::max(1, std::min(sv->opts.max_active_ctas, std::max(1, sv->ctx->sm_count)));
    if (!b->mm) return cap;
    return std::max(1, cap / (b->m * mm_cluster_ctas(ilog2i(b->nt))));
}

// a bucket's own table set: a problem with this shape's grid (zero tables),
// so free slots always point at live twiddles
int srv_bucket_tables(fl_server* sv, SrvBucket* b) {
    const int nt = b->nt, m = b->m;
    std::vector<double> D((size_t)nt * m, 0.0), g((size_t)m * m * m * m, 0.0), h(2 * (size_t)nt, 0.0),
        ss(nt, 1.0);
    for (int i = 0; i < m; i++) g[i + m * (i + m * (i + m * i))] = 1.0;
    return fl_problem_create(sv->ctx, nt, m, D.data(), g.data(), h.data(), ss.data(), 1.0, 1.0,
                             1e-8, 1e-6, b->precision, &b->tables);
}

int srv_new_chunk(fl_server* sv, SrvBucket* b) {
    fl_ctx* ctx = sv->ctx;
    auto c = std::make_unique<SrvChunk>();
    c->mm = b->mm;
    c->B = srv_chunk_slots(sv, b);
    const size_t need = srv_slot_bytes(sv, b->tables) * c->B;
    if (sv->opts.hbm_budget_bytes && sv->hbm_used + need > sv->opts.hbm_budget_bytes) {
        // a smaller chunk if at least one slot fits
        const size_t one = srv_slot_bytes(sv, b->tables);
        const size_t left = sv->opts.hbm_budget_bytes - std::min(sv->hbm_used, sv->opts.hbm_budget_bytes);
        c->B = (int)std::min<size_t>(c->B, left / one);
        if (c->B < 1) return FL_OOM_ADMISSION;
    }
    CU(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming));
    fl_ctx_opts o = sv->wopts;
    o.hbm_budget_bytes = 0;
    int rc = c->mm ? mm_work_create(b->tables, c->B, 0, MODE_FORWARD, 0, &c->mw, &o, c->stream)
                   : work_create(b->tables, c->B, 0, MODE_FORWARD, &c->w, &o, c->stream);
    if (rc) return rc;
    CU(cudaMalloc(&c->d_masks, (size_t)c->B * b->nt));
    // every slot starts free (finished)
    if (c->mm) {
        std::vector<MmState> st(c->B);
        for (auto& x : st) {
            memset(&x, 0, sizeof x);
            x.phase = PH_DONE;
        }
        CU(cudaMemcpyAsync(c->mw->d_state, st.data(), sizeof(MmState) * c->B,
                           cudaMemcpyHostToDevice, c->stream));
    } else {
        std::vector<SlotState> st(c->B);
        for (auto& x : st) {
            memset(&x, 0, sizeof x);
            x.phase = PH_DONE;
        }
        CU(cudaMemcpyAsync(c->w->d_state, st.data(), sizeof(SlotState) * c->B,
                           cudaMemcpyHostToDevice, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    c->slot.assign(c->B, nullptr);
    c->bytes = (c->mm ? c->mw->pool_bytes : c->w->pool_bytes) + (size_t)c->B * b->nt;
    sv->hbm_used += c->bytes;
    b->chunks.push_back(c.release());
    return FL_OK;
}

// place request r into free slot i of chunk c (stream-ordered before the next launch)
int srv_admit(fl_server* sv, SrvBucket* b, SrvChunk* c, int i, SrvRequest* r) {
    Nvtx nvtx_("fl: server admit");
    fl_ctx* ctx = sv->ctx;
    const fl_problem* pr = r->prob;
    const size_t nm = (size_t)b->nt * b->m;
    const int mode = r->kind == FL_REQ_BAND_GRADIENT ? MODE_BAND_GRADIENT : MODE_FORWARD;
    unsigned char* dmask = c->d_masks + (size_t)i * b->nt;
    if (!r->mask.empty())
        CU(cudaMemcpyAsync(dmask, r->mask.data(), b->nt, cudaMemcpyHostToDevice, c->stream));
    if (c->mm) {
        MmDesc& d = c->mw->h_desc[i];
        d.Dturns = pr->d_Dturns;
        for (int q = 0; q < 2; q++) {
            d.Heff[q] = pr->d_Heff[q];
            d.ss[q] = pr->d_ss[q];
            d.G[q] = pr->d_G[q];
        }
        d.Ga = pr->d_Ga;
        d.Gtc = pr->d_Gtc;
        d.Gtcs = pr->d_Gtcs;
        d.rank = pr->rank;
        d.Vz = pr->d_Vz;
        d.Utc = pr->d_Utc;
        d.Utcs = pr->d_Utcs;
        d.one_m_fR = pr->one_m_fR;
        d.L = r->L;
        d.reltol = pr->reltol;
        d.abstol = pr->abstol;
        d.mode = mode;
        d.log_cost = r->log_cost;
        d.objective = r->objective;
        d.obj_tau = r->obj_tau;
        d.phase_per_mode = 0;
        d.mask = dmask;
        // a forward-only request keeps no checkpoints or step log
        d.ck_cap = mode == MODE_FORWARD ? 0 : c->mw->K;
        d.step_cap = mode == MODE_FORWARD ? 0 : c->mw->stepcap;
        CU(cudaMemcpyAsync((double*)d.u0, r->u0.data(), 16 * nm, cudaMemcpyHostToDevice, c->stream));
        CU(cudaMemcpyAsync((MmDesc*)c->mw->d_desc + i, &d, sizeof(MmDesc), cudaMemcpyHostToDevice,
                           c->stream));
        CU(cudaMemsetAsync(c->mw->d_state + i, 0, sizeof(MmState), c->stream));
    } else {
        SlotDesc& d = reinterpret_cast<SlotDesc*>(c->w->h_desc.data())[i];
        d.Dturns = pr->d_Dturns;
        for (int q = 0; q < 2; q++) {
            d.Heff[q] = pr->d_Heff[q];
            d.ss[q] = pr->d_ss[q];
        }
        d.gamma = pr->gamma0;
        d.one_m_fR = pr->one_m_fR;
        d.L = r->L;
        d.reltol = pr->reltol;
        d.abstol = pr->abstol;
        d.mode = mode;
        d.log_cost = r->log_cost;
        d.objective = r->objective;
        d.obj_tau = r->obj_tau;
        d.mask = dmask;
        // a forward-only request keeps no checkpoints or step log
        d.ck_cap = mode == MODE_FORWARD ? 0 : c->w->K;
        d.step_cap = mode == MODE_FORWARD ? 0 : c->w->stepcap;
        CU(cudaMemcpyAsync((double*)d.u0, r->u0.data(), 16 * nm, cudaMemcpyHostToDevice, c->stream));
        CU(cudaMemcpyAsync((SlotDesc*)c->w->d_desc + i, &d, sizeof(SlotDesc), cudaMemcpyHostToDevice,
                           c->stream));
        CU(cudaMemsetAsync(c->w->d_state + i, 0, sizeof(SlotState), c->stream));
    }
    c->slot[i] = r;
    return FL_OK;
}

// after a launch: copy finished requests' results out and free their slots
// (the status is published under the server lock by the caller)
int srv_retire(fl_server* sv, SrvBucket* b, SrvChunk* c,
               std::vector<std::pair<SrvRequest*, int>>& done) {
    Nvtx nvtx_("fl: server retire");
    fl_ctx* ctx = sv->ctx;
    const size_t nm = (size_t)b->nt * b->m;
    if (c->mm) {
        c->hms.resize(c->B);
        CU(cudaMemcpyAsync(c->hms.data(), c->mw->d_state, sizeof(MmState) * c->B,
                           cudaMemcpyDeviceToHost, c->stream));
    } else {
        c->hs.resize(c->B);
        CU(cudaMemcpyAsync(c->hs.data(), c->w->d_state, sizeof(SlotState) * c->B,
                           cudaMemcpyDeviceToHost, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < c->B; i++) {
        SrvRequest* r = c->slot[i];
        if (!r) continue;
        const int ph = c->mm ? c->hms[i].phase : c->hs[i].phase;
        if (ph != PH_DONE) continue;
        int st;
        if (c->mm) {
            mm_fill_stats(c->hms[i], &r->stats);
            st = c->hms[i].status;
            r->J = c->hms[i].J;
        } else {
            fill_stats(c->hs[i], &r->stats);
            st = c->hs[i].status;
            r->J = c->hs[i].J;
        }
        if (st == ST_OK) {
            const double* uL = c->mm ? c->mw->h_desc[i].uL_out
                                     : reinterpret_cast<SlotDesc*>(c->w->h_desc.data())[i].uL_out;
            const double* gr = c->mm ? c->mw->h_desc[i].grad_out
                                     : reinterpret_cast<SlotDesc*>(c->w->h_desc.data())[i].grad_out;
            if (r->kind == FL_REQ_FORWARD && r->out_field)
                CU(cudaMemcpyAsync(r->out_field, uL, 16 * nm, cudaMemcpyDeviceToHost, c->stream));
            if (r->kind == FL_REQ_BAND_GRADIENT && r->out_grad)
                CU(cudaMemcpyAsync(r->out_grad, gr, 8 * (size_t)b->nt, cudaMemcpyDeviceToHost,
                                   c->stream));
        }
        c->slot[i] = nullptr;
        done.emplace_back(r, st);
    }
    CU(cudaStreamSynchronize(c->stream));
    return FL_OK;
}

int srv_launch(fl_server* sv, SrvBucket* b, SrvChunk* c) {
    Nvtx nvtx_("fl: server launch");
    fl_ctx* ctx = sv->ctx;
    const int logn = ilog2i(b->nt);
    if (c->mm) {
        MmRound a{};
        a.desc = c->mw->d_desc;
        a.state = c->mw->d_state;
        a.active = c->mw->d_active;
        a.nactive = c->B;
        a.M = b->m;
        a.NP = c->mw->np;
        a.N = b->nt;
        a.fp64 = b->precision == FL_PRECISION_FP64;
        a.control = 1;
        a.tensor_cores = 1;
        a.ndone = nullptr;
        a.stream = c->stream;
        MmRoundFn round = mm_round_launcher(logn);
        // control (prepares newly admitted slots, idempotent for the rest) and
        // evals_per_launch rounds over all the chunk's slots (finished ones are
        // skipped by the kernels): the same launches every time, so they are
        // captured once per chunk as a CUDA graph and replayed
        if (!c->graph) {
            cudaGraph_t g = nullptr;
            CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e1 = mm_launch_control(a, 0);
            for (int r = 0; e1 == cudaSuccess && r < sv->opts.evals_per_launch; r++) e1 = round(a);
            const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
            if (e1 != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                return set_err(ctx, FL_ECUDA, "capturing a server launch: %s",
                               cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            }
            const cudaError_t e3 = cudaGraphInstantiate(&c->graph, g, 0);
            cudaGraphDestroy(g);
            if (e3 != cudaSuccess) {
                c->graph = nullptr;
                return set_err(ctx, FL_ECUDA, "instantiating a server launch: %s",
                               cudaGetErrorString(e3));
            }
        }
        CU(cudaGraphLaunch(c->graph, c->stream));
        sv->launches += 1 + (long)sv->opts.evals_per_launch * (a.fp64 ? 7 : 10);
    } else {
        LaunchFn fn = sm_launcher(b->precision == FL_PRECISION_FP64, logn);
        LaunchArgs a{c->w->d_desc, c->w->d_state, c->w->d_active, c->B,
                     sv->opts.evals_per_launch, c->stream};
        CU(fn(a));
        sv->launches++;
    }
    CU(cudaEventRecord(c->ev, c->stream));
    c->inflight = true;
    return FL_OK;
}

SrvBucket* srv_bucket_for(fl_server* sv, const fl_problem* pr) {
    for (auto* b : sv->buckets)
        if (b->nt == pr->nt && b->m == pr->m && b->precision == pr->precision) return b;
    return nullptr;
}

SrvBucket* srv_bucket_get(fl_server* sv, const fl_problem* pr, int& rc) {
    rc = FL_OK;
    SrvBucket* b = srv_bucket_for(sv, pr);
    if (b) return b;
    b = new SrvBucket();
    b->nt = pr->nt;
    b->m = pr->m;
    b->precision = pr->precision;
    b->mm = pr->use_mm;
    sv->buckets.push_back(b);
    rc = srv_bucket_tables(sv, b);
    return b;
}

// One pass: retire finished launches, admit waiting requests in arrival
// order while the requests in flight fit the SMs (and the HBM budget allows
// their slots), launch every chunk with work.  Returns whether anything
// happened.
int srv_progress(fl_server* sv, bool& did) {
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        while (!sv->incoming.empty()) {
            sv->waiting.push_back(sv->incoming.front());
            sv->incoming.pop_front();
            did = true;
        }
    }
    std::vector<std::pair<SrvRequest*, int>> done;
    for (auto* b : sv->buckets)
        for (auto* c : b->chunks) {
            if (!c->inflight) continue;
            const cudaError_t q = cudaEventQuery(c->ev);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) {
                fl_ctx* ctx = sv->ctx;
                CU(q);
            }
            c->inflight = false;
            const size_t before = done.size();
            int rc = srv_retire(sv, b, c, done);
            if (rc) return rc;
            for (size_t k = before; k < done.size(); k++) sv->active_w -= done[k].first->weight;
            did = true;
        }
    const long cap = sv->opts.max_active_ctas;
    while (!sv->waiting.empty()) {
        SrvRequest* r = sv->waiting.front();
        if (sv->active_w > 0 && sv->active_w + r->weight > cap) break;
        int rc;
        SrvBucket* b = srv_bucket_get(sv, r->prob, rc);
        if (rc) return rc;
        SrvChunk* fc = nullptr;
        int fi = -1;
        for (auto* c : b->chunks) {
            for (int i = 0; i < c->B && fi < 0; i++)
                if (!c->slot[i]) {
                    fc = c;
                    fi = i;
                }
            if (fc) break;
        }
        if (!fc) {
            rc = srv_new_chunk(sv, b);
            if (rc == FL_OOM_ADMISSION) break;  // wait for slots to free up
            if (rc) return rc;
            fc = b->chunks.back();
            fi = 0;
        }
        rc = srv_admit(sv, b, fc, fi, r);
        if (rc) return rc;
        sv->active_w += r->weight;
        sv->waiting.pop_front();
        did = true;
    }
    sv->n_waiting.store((long)sv->waiting.size());
    for (auto* b : sv->buckets)
        for (auto* c : b->chunks) {
            if (c->inflight) continue;
            bool any = false;
            for (auto* r : c->slot) any |= r != nullptr;
            if (!any) continue;
            int rc = srv_launch(sv, b, c);
            if (rc) return rc;
            did = true;
        }
    if (!done.empty()) {
        const double t = now_ms();
        std::lock_guard<std::mutex> lk(sv->mu);
        for (auto& rs : done) {
            rs.first->t_done = t;
            rs.first->status = rs.second;
            sv->completed++;
        }
        sv->cv.notify_all();
    }
    return FL_OK;
}

void srv_thread(fl_server* sv) {
    cudaSetDevice(sv->ctx->device);
    while (!sv->stop.load()) {
        bool did = false;
        const int rc = srv_progress(sv, did);
        if (rc) {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->fatal = rc;
            sv->err = sv->ctx->err;
            for (auto& kv : sv->reqs)
                if (kv.second->status == FL_EBUSY) kv.second->status = rc;
            sv->cv.notify_all();
            return;
        }
        if (!did) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

}  // namespace

extern "C" {

const char* fl_version(void) { return "fiberlab-gpu 0.1 (sm_100a)"; }

const char* fl_status_string(int s) {
    switch (s) {
        case FL_OK: return "ok";
        case FL_EINVAL: return "invalid argument";
        case FL_NONFINITE: return "non-finite value in the solution";
        case FL_DT_UNDERFLOW: return "step size below floating-point resolution";
        case FL_MAXITERS: return "maximum attempted steps reached";
        case FL_ENOMEM: return "device out of memory";
        case FL_NONSYMMETRIC: return "adjoint requires a permutation-symmetric gamma tensor";
        case FL_ENODEV: return "no usable CUDA device";
        case FL_ECUDA: return "CUDA runtime error";
        case FL_ECAPACITY: return "checkpoint / segment / step-log capacity exceeded";
        case FL_EUNSUPPORTED: return "unsupported shape";
        case FL_OOM_ADMISSION: return "request exceeds the HBM budget";
        case FL_EBUSY: return "request not finished";
        case FL_TIMEOUT: return "wait limit reached";
        case FL_ECHECK: return "checked build: a solver index left its buffer's bounds";
        default: return "unknown status";
    }
}

int fl_ctx_create(int device, const fl_ctx_opts* opts, fl_ctx** out) {
    if (!out) return FL_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) return FL_ENODEV;
    fl_ctx* ctx = new (std::nothrow) fl_ctx();
    if (!ctx) return FL_ENOMEM;
    ctx->device = device;
    ctx->opts.hbm_budget_bytes = 0;
    ctx->opts.checkpoints = 32;
    ctx->opts.segment_steps = 64;
    ctx->opts.step_log = 0;  // one entry per allowed attempted step
    ctx->opts.max_iters = 100000;
    if (opts) {
        if (opts->hbm_budget_bytes) ctx->opts.hbm_budget_bytes = opts->hbm_budget_bytes;
        if (opts->checkpoints) ctx->opts.checkpoints = opts->checkpoints;
        if (opts->segment_steps) ctx->opts.segment_steps = opts->segment_steps;
        if (opts->step_log) ctx->opts.step_log = opts->step_log;
        if (opts->max_iters) ctx->opts.max_iters = opts->max_iters;
    }
    if (!pow2(ctx->opts.checkpoints) || ctx->opts.checkpoints < 2 ||
        ctx->opts.segment_steps < 1 || ctx->opts.step_log < 0 || ctx->opts.max_iters < 1) {
        delete ctx;
        return FL_EINVAL;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return FL_ENODEV;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        delete ctx;
        return FL_ENODEV;
    }
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return FL_ECUDA;
    }
    ctx->stream = ctx->own;
    for (auto& e : ctx->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            fl_ctx_destroy(ctx);
            return FL_ECUDA;
        }
    *out = ctx;
    return FL_OK;
}

int fl_ctx_destroy(fl_ctx* ctx) {
    if (!ctx) return FL_EINVAL;
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return FL_OK;
}

int fl_ctx_set_stream(fl_ctx* ctx, void* stream) {
    if (!ctx) return FL_EINVAL;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    // work already queued on the previous stream completes before the switch,
    // so the context's device buffers are never used by two streams at once
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
    return FL_OK;
}

void* fl_ctx_get_stream(const fl_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

const char* fl_last_error(const fl_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

long fl_ctx_launch_count(const fl_ctx* ctx) { return ctx ? ctx->launches : 0; }

int fl_ctx_timing(const fl_ctx* ctx, double* last_call_ms, double* last_kernel_ms) {
    if (!ctx) return FL_EINVAL;
    if (last_call_ms) *last_call_ms = ctx->call_ms;
    if (last_kernel_ms) *last_kernel_ms = ctx->kernel_ms;
    return FL_OK;
}

int fl_ctx_synchronize(fl_ctx* ctx) {
    if (!ctx) return FL_EINVAL;
    CU(cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

int fl_problem_create(fl_ctx* ctx, int nt, int m, const double* D, const double* gamma,
                      const double* hR, const double* selfsteep, double one_m_fR, double L,
                      double reltol, double abstol, int precision, fl_problem** out) {
    if (!ctx || !out) return FL_EINVAL;
    *out = nullptr;
    if (nt < 4 || !pow2(nt)) return set_err(ctx, FL_EINVAL, "Nt must be a power of two >= 4");
    if (m < 1) return set_err(ctx, FL_EINVAL, "M must be a positive integer");
    if (!D || !gamma || !hR || !selfsteep) return set_err(ctx, FL_EINVAL, "null table");
    if (precision != FL_PRECISION_FP32 && precision != FL_PRECISION_FP64)
        return set_err(ctx, FL_EINVAL, "unknown precision %d", precision);
    if (!(std::isfinite(L) && L > 0)) return set_err(ctx, FL_EINVAL, "L must be positive and finite");
    if (!(std::isfinite(reltol) && reltol > 0))
        return set_err(ctx, FL_EINVAL, "reltol must be positive and finite");
    if (!(std::isfinite(abstol) && abstol > 0))
        return set_err(ctx, FL_EINVAL, "abstol must be positive and finite");
    if (!std::isfinite(one_m_fR)) return set_err(ctx, FL_EINVAL, "one_m_fR must be finite");
    const long m4 = (long)m * m * m * m;
    for (long i = 0; i < m4; i++)
        if (!std::isfinite(gamma[i])) return set_err(ctx, FL_EINVAL, "gamma tensor must be finite");
    for (long i = 0; i < (long)nt * m; i++)
        if (!std::isfinite(D[i])) return set_err(ctx, FL_EINVAL, "dispersion must be finite");
    for (int i = 0; i < 2 * nt; i++)
        if (!std::isfinite(hR[i])) return set_err(ctx, FL_EINVAL, "Raman response must be finite");
    for (int i = 0; i < nt; i++)
        if (!std::isfinite(selfsteep[i])) return set_err(ctx, FL_EINVAL, "selfsteep must be finite");
    if (!hermitian(hR, nt))
        return set_err(ctx, FL_EINVAL, "Raman response spectrum must be Hermitian");
    auto pr = std::make_unique<fl_problem>();
    pr->ctx = ctx;
    pr->nt = nt;
    pr->m = m;
    pr->precision = precision;
    pr->one_m_fR = one_m_fR;
    pr->L = L;
    pr->reltol = reltol;
    pr->abstol = abstol;
    pr->gamma0 = gamma[0];
    pr->gamma_sym = gamma_symmetric(gamma, m);
    // the single-CTA stepper covers M = 1 up to 2^14 (FP32 mode) / 2^13 (FP64
    // mode); larger transforms run on the multimode runtime's kernels
    pr->use_mm = m > 1 || ilog2i(nt) > (precision == FL_PRECISION_FP64 ? 13 : 14);
    if (pr->use_mm ? ((m > 1 && !mm_supported_modes(m)) || !mm_round_launcher(ilog2i(nt)))
                   : !sm_launcher(precision == FL_PRECISION_FP64, ilog2i(nt)))
        return set_err(ctx, FL_EUNSUPPORTED, "built shapes: M = 1 with Nt = 2^6..2^15, "
                       "M = 2..10 with Nt = 2^6..2^15 (got M = %d, Nt = %d)", m, nt);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    int rc = upload_tables(pr.get(), D, hR, selfsteep);
    if (!rc && pr->use_mm) rc = mm_upload_G(pr.get(), gamma);
    if (rc) {
        fl_problem_destroy(pr.release());
        return rc;
    }
    *out = pr.release();
    return FL_OK;
}

int fl_problem_set_objective(fl_problem* pr, int objective, double worst_mode_tau) {
    int rc = check_problem(pr);
    if (rc) return rc;
    if (objective < FL_OBJ_RAMAN_BAND || objective > FL_OBJ_RAMAN_PEAK)
        return set_err(pr->ctx, FL_EINVAL, "unknown objective %d", objective);
    if (!(std::isfinite(worst_mode_tau) && worst_mode_tau > 0))
        return set_err(pr->ctx, FL_EINVAL, "worst-mode smoothness tau must be positive and finite");
    pr->objective = objective;
    pr->obj_tau = worst_mode_tau;
    return FL_OK;
}

int fl_problem_destroy(fl_problem* pr) {
    if (!pr) return FL_EINVAL;
    delete pr->last;
    delete pr->mlast;
    cudaFree(pr->d_stage);
    cudaFree(pr->d_ev);
    cudaFree(pr->d_G[0]);
    cudaFree(pr->d_G[1]);
    cudaFree(pr->d_Ga);
    cudaFree(pr->d_Gtc);
    cudaFree(pr->d_Gtcs);
    cudaFree(pr->d_Vz);
    cudaFree(pr->d_Utc);
    cudaFree(pr->d_Utcs);
    cudaFree(pr->d_Dturns);
    for (int q = 0; q < 2; q++) {
        cudaFree(pr->d_Heff[q]);
        cudaFree(pr->d_ss[q]);
        cudaFree(pr->d_tw[q]);
    }
    delete pr;
    return FL_OK;
}

int fl_forward_gain(fl_problem* pr, const fl_gain* gain, double pump_power, const double* u0,
                    const double* saveat, int nsave, double* out_spectra, double* out_pump,
                    fl_stats* stats) {
    Nvtx nvtx_("fl_forward_gain");
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!gain || !u0 || !saveat || !out_spectra || !out_pump)
        return set_err(ctx, FL_EINVAL, "null argument");
    // propagation.jl:60-70: sorted, unique, starts at 0 and ends at L
    if (nsave < 2) return set_err(ctx, FL_EINVAL, "saveat must include 0 and the fiber length");
    for (int i = 0; i < nsave; i++) {
        if (!std::isfinite(saveat[i])) return set_err(ctx, FL_EINVAL, "saveat distances must be finite");
        if (i > 0 && !(saveat[i] > saveat[i - 1]))
            return set_err(ctx, FL_EINVAL, "saveat distances must be sorted and unique");
    }
    if (saveat[0] != 0.0 || saveat[nsave - 1] != pr->L)
        return set_err(ctx, FL_EINVAL, "saveat must start at 0 and end at the fiber length");
    const int nt = pr->nt, logn = ilog2i(nt);
    if (pr->m != 1 || pr->precision != FL_PRECISION_FP32 || !gain_built(logn))
        return set_err(ctx, FL_EUNSUPPORTED,
                       "gain propagation is built for M = 1 in FP32 mode at Nt = 2^6..2^13");
    if (gain->kind != FL_GAIN_CONSTANT && gain->kind != FL_GAIN_YDFA)
        return set_err(ctx, FL_EINVAL, "unknown gain model %d", gain->kind);
    if (!std::isfinite(pump_power)) return set_err(ctx, FL_EINVAL, "pump power must be finite");
    // the gain tables: W12/W21 weights and the g(ω) coefficients per bin
    std::vector<double> tab(4 * (size_t)nt, 0.0);
    double r12c = 0, r21c = 0, inv_tau = 0, gpe = 0, gpa = 0;
    if (gain->kind == FL_GAIN_CONSTANT) {
        if (!std::isfinite(gain->g_const)) return set_err(ctx, FL_EINVAL, "gain must be finite");
    } else {
        const fl_gain& g = *gain;
        if (!g.sigma_as || !g.sigma_es || !g.h_nu_s)
            return set_err(ctx, FL_EINVAL, "YDFA gain needs the per-bin cross sections");
        const double sc[] = {g.gamma_p, g.sigma_ap, g.sigma_ep, g.h_nu_p, g.gamma_s, g.area,
                             g.rho, g.tau21, g.psd_scale, g.df};
        for (double x : sc)
            if (!(std::isfinite(x) && x >= 0)) return set_err(ctx, FL_EINVAL, "YDFA parameters must be finite and nonnegative");
        if (!(g.h_nu_p > 0 && g.area > 0 && g.tau21 > 0))
            return set_err(ctx, FL_EINVAL, "YDFA photon energy, area and lifetime must be positive");
        for (int b = 0; b < nt; b++) {
            if (!(std::isfinite(g.sigma_as[b]) && g.sigma_as[b] >= 0 && std::isfinite(g.sigma_es[b]) &&
                  g.sigma_es[b] >= 0 && g.h_nu_s[b] > 0 && std::isfinite(g.h_nu_s[b])))
                return set_err(ctx, FL_EINVAL, "YDFA cross sections and photon energies must be finite");
            const double w = g.gamma_s * g.psd_scale * g.df / (g.h_nu_s[b] * g.area);
            tab[b] = w * g.sigma_as[b];                      // W12 weight
            tab[nt + b] = w * g.sigma_es[b];                 // W21 weight
            tab[2 * (size_t)nt + b] = g.gamma_s * g.sigma_as[b] * g.rho;  // sA
            tab[3 * (size_t)nt + b] = g.gamma_s * g.sigma_es[b] * g.rho;  // sE
        }
        r12c = g.gamma_p * g.sigma_ap / (g.h_nu_p * g.area);
        r21c = g.gamma_p * g.sigma_ep / (g.h_nu_p * g.area);
        inv_tau = 1.0 / g.tau21;
        gpe = g.gamma_p * g.sigma_ep * g.rho;
        gpa = g.gamma_p * g.sigma_ap * g.rho;
    }
    double nrm = 0.0;
    for (int i = 0; i < 2 * nt; i++) {
        if (!std::isfinite(u0[i])) return set_err(ctx, FL_EINVAL, "input spectrum must be finite");
        nrm += u0[i] * u0[i];
    }
    if (!(nrm > 0)) return set_err(ctx, FL_EINVAL, "input spectrum must be nonzero");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    // one device area: launch, two states, seven FP32 stages, two scratch
    // fields, error partial and weights, output, gain tables, descriptor, result
    // (the size is the sum of the regions taken below, each rounded up to the
    // 256-byte alignment that take() gives it)
    const size_t F = 16 * (size_t)nt, H = 8 * (size_t)nt;
    auto al = [](size_t n) { return (n + 255) & ~size_t(255); };
    const size_t bytes = 4 * al(F) + 7 * al(H) + 2 * al(F) + al(F) + al(H) + al(4 * H) +
                         al(8 * (size_t)nsave) + al(F * (size_t)nsave) + al(8 * (size_t)nsave) +
                         al(sizeof(GainDesc)) + al(sizeof(GainOut));
    char* pool = nullptr;
    CU(cudaMalloc(&pool, bytes));
    char* p = pool;
    auto take = [&](size_t n) { char* q = p; p += al(n); return q; };
    GainDesc hd;
    memset(&hd, 0, sizeof hd);
    SlotDesc& d = hd.s;
    d.Dturns = pr->d_Dturns;
    d.Heff[0] = pr->d_Heff[0];
    d.ss[0] = pr->d_ss[0];
    d.tw[0] = pr->d_tw[0];   // FP32 twiddles only (no FP64 stage here)
    d.gamma = pr->gamma0;
    d.one_m_fR = pr->one_m_fR;
    d.L = pr->L;
    d.reltol = pr->reltol;
    d.abstol = pr->abstol;
    d.mode = MODE_FORWARD;
    d.max_iters = ctx->opts.max_iters;
    double* d_u0 = (double*)take(F);
    d.u0 = d_u0;
    d.u[0] = (double*)take(F);
    d.u[1] = (double*)take(F);
    d.uL_out = (double*)take(F);
    for (int i = 0; i < 7; i++) d.kf[i] = take(H);
    d.scr[0] = take(F);
    d.scr[1] = take(F);
    d.esv = (double*)take(F);
    d.skv = (double*)take(H);
    double* d_tab = (double*)take(4 * H);
    double* d_zsave = (double*)take(8 * (size_t)nsave);
    d.zsave = d_zsave;
    d.nsave = nsave;
    d.save_out = (double*)take(F * (size_t)nsave);
    hd.pump_save = (double*)take(8 * (size_t)nsave);
    hd.kind = gain->kind;
    hd.g_const = gain->g_const;
    hd.r12c = r12c;
    hd.r21c = r21c;
    hd.inv_tau = inv_tau;
    hd.gpe = gpe;
    hd.gpa = gpa;
    hd.wa = d_tab;
    hd.we = d_tab + nt;
    hd.sA = d_tab + 2 * (size_t)nt;
    hd.sE = d_tab + 3 * (size_t)nt;
    hd.pump0 = pump_power;
    GainDesc* d_desc = (GainDesc*)take(sizeof(GainDesc));
    GainOut* d_out = (GainOut*)take(sizeof(GainOut));
    if ((size_t)(p - pool) > bytes) {
        cudaFree(pool);
        return set_err(ctx, FL_ECUDA, "internal: gain workspace overflow (%zu > %zu)",
                       (size_t)(p - pool), bytes);
    }
    GainOut ho{};
    cudaError_t e = cudaMemcpyAsync(d_u0, u0, F, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_tab, tab.data(), 4 * H, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_zsave, saveat, 8 * (size_t)nsave, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_desc, &hd, sizeof hd, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[0], ctx->stream);
    if (e == cudaSuccess) e = launch_gain(logn, d_desc, d_out, ctx->stream);
    if (e == cudaSuccess) ctx->launches++;
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[1], ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&ho, d_out, sizeof ho, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out_spectra, d.save_out, F * (size_t)nsave, cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out_pump, hd.pump_save, 8 * (size_t)nsave, cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(pool);
    if (e != cudaSuccess) return set_err(ctx, FL_ECUDA, "gain propagation: %s", cudaGetErrorString(e));
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->naccept = ho.naccept;
        stats->nreject = ho.nreject;
        stats->nf = ho.nf;
        stats->status = ho.status;
        stats->z_end = ho.z_end;
    }
    if (ho.status) return set_err(ctx, ho.status, "%s", fl_status_string(ho.status));
    return FL_OK;
}

int fl_forward(fl_problem* pr, const double* u0, const double* saveat, int nsave,
               double* out_spectra, fl_stats* stats) {
    Nvtx nvtx_("fl_forward");
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!u0 || nsave < 0 || (nsave > 0 && (!saveat || !out_spectra)))
        return set_err(ctx, FL_EINVAL, "null argument");
    // propagation.jl:60-70: sorted, unique, starts at 0 and ends at L
    if (nsave > 0) {
        if (nsave < 2) return set_err(ctx, FL_EINVAL, "saveat must include 0 and the fiber length");
        for (int i = 0; i < nsave; i++)
            if (!std::isfinite(saveat[i])) return set_err(ctx, FL_EINVAL, "saveat distances must be finite");
        for (int i = 1; i < nsave; i++)
            if (!(saveat[i] > saveat[i - 1]))
                return set_err(ctx, FL_EINVAL, "saveat distances must be sorted and unique");
        if (saveat[0] != 0.0 || saveat[nsave - 1] != pr->L)
            return set_err(ctx, FL_EINVAL, "saveat must start at 0 and end at the fiber length");
    }
    const int nt = pr->nt;
    double nrm = 0.0;
    for (int i = 0; i < 2 * nt * pr->m; i++) {
        if (!std::isfinite(u0[i])) return set_err(ctx, FL_EINVAL, "input spectrum must be finite");
        nrm += u0[i] * u0[i];
    }
    if (!(nrm > 0)) return set_err(ctx, FL_EINVAL, "input spectrum must be nonzero");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    if (pr->use_mm) return mm_forward(pr, u0, saveat, nsave, out_spectra, stats);
    // the problem's one-slot forward workspace is reused by later forwards
    // with the same number of save positions (no allocation per call)
    Work* w = pr->last;
    if (w && w->B == 1 && w->nsave == nsave) {
        rc = set_mode(ctx, w, MODE_FORWARD, 0);
        if (rc) return rc;
        CU(cudaMemsetAsync(w->d_state, 0, sizeof(SlotState), ctx->stream));
    } else {
        delete pr->last;
        pr->last = nullptr;
        w = nullptr;
        rc = new_work(pr, 1, nsave, MODE_FORWARD, &w);
        if (rc) return rc;
        pr->last = w;
    }
    CU(cudaMemcpyAsync(w->d_u0, u0, 16 * (size_t)nt, cudaMemcpyHostToDevice, ctx->stream));
    if (nsave)
        CU(cudaMemcpyAsync(w->d_zsave, saveat, 8 * (size_t)nsave, cudaMemcpyHostToDevice,
                           ctx->stream));
    rc = run_to_completion(pr, w);
    if (rc) return rc;
    std::vector<SlotState> st;
    rc = read_states(ctx, w, st);
    if (rc) return rc;
    if (stats) fill_stats(st[0], stats);
    if (st[0].status) return set_err(ctx, st[0].status, "%s", fl_status_string(st[0].status));
    if (nsave)
        CU(cudaMemcpy(out_spectra, w->d_save, 16 * (size_t)nt * nsave, cudaMemcpyDeviceToHost));
    return FL_OK;
}

int fl_adjoint(fl_problem* pr, const double* lambdaL, double* lambda0, fl_stats* stats) {
    Nvtx nvtx_("fl_adjoint");
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!lambdaL || !lambda0) return set_err(ctx, FL_EINVAL, "null argument");
    if (!pr->gamma_sym)
        return set_err(ctx, FL_NONSYMMETRIC,
                       "fiber adjoint requires a fully permutation-symmetric gamma tensor");
    if (!(pr->use_mm ? (void*)pr->mlast : (void*)pr->last))
        return set_err(ctx, FL_EINVAL, "fl_adjoint needs a preceding fl_forward");
    const int nt = pr->nt;
    for (int i = 0; i < 2 * nt * pr->m; i++)
        if (!std::isfinite(lambdaL[i]))
            return set_err(ctx, FL_EINVAL, "adjoint terminal condition must be finite");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    if (pr->use_mm) return mm_adjoint(pr, lambdaL, lambda0, stats);
    Work* w = pr->last;
    std::vector<SlotState> st;
    rc = read_states(ctx, w, st);
    if (rc) return rc;
    if (st[0].phase != PH_DONE || st[0].status != ST_OK)
        return set_err(ctx, FL_EINVAL, "the last forward did not complete");
    st[0].phase = PH_SEED;
    CU(cudaMemcpyAsync(w->d_state, st.data(), sizeof(SlotState), cudaMemcpyHostToDevice,
                       ctx->stream));
    rc = set_mode(ctx, w, MODE_SEEDED_ADJOINT, 0);
    if (rc) return rc;
    CU(cudaMemcpyAsync(w->d_lamL, lambdaL, 16 * (size_t)nt, cudaMemcpyHostToDevice, ctx->stream));
    rc = run_to_completion(pr, w);
    if (rc) return rc;
    rc = read_states(ctx, w, st);
    if (rc) return rc;
    if (stats) fill_stats(st[0], stats);
    if (st[0].status) return set_err(ctx, st[0].status, "%s", fl_status_string(st[0].status));
    CU(cudaMemcpy(lambda0, w->d_lam0, 16 * (size_t)nt, cudaMemcpyDeviceToHost));
    return FL_OK;
}

int fl_forward_times(fl_problem* pr, double* t_out, long cap, long* n_out) {
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!n_out || (cap > 0 && !t_out)) return set_err(ctx, FL_EINVAL, "null argument");
    if (!(pr->use_mm ? (void*)pr->mlast : (void*)pr->last))
        return set_err(ctx, FL_EINVAL, "fl_forward_times needs a preceding fl_forward");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    // the accepted-step log (z_n, dt_n) of slot 0 and its final position
    long nsteps = 0;
    double zend = 0.0;
    const double* d_log = nullptr;
    if (pr->use_mm) {
        std::vector<MmState> st;
        rc = mm_read_states(ctx, pr->mlast, 1, st);
        if (rc) return rc;
        if (st[0].status != ST_OK || st[0].nsteps <= 0)
            return set_err(ctx, FL_EINVAL, "the last forward did not complete");
        nsteps = st[0].nsteps;
        zend = st[0].z;
        d_log = pr->mlast->h_desc[0].steplog;
    } else {
        std::vector<SlotState> st;
        rc = read_states(ctx, pr->last, st);
        if (rc) return rc;
        if (st[0].status != ST_OK || st[0].nsteps <= 0)
            return set_err(ctx, FL_EINVAL, "the last forward did not complete");
        nsteps = st[0].nsteps;
        zend = st[0].z;
        d_log = reinterpret_cast<const SlotDesc*>(pr->last->h_desc.data())[0].steplog;
    }
    *n_out = nsteps + 1;
    if (cap <= 0) return FL_OK;
    std::vector<double> lg(2 * (size_t)nsteps);
    CU(cudaMemcpyAsync(lg.data(), d_log, sizeof(double) * lg.size(), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (long i = 0; i < nsteps && i < cap; i++) t_out[i] = lg[2 * i];
    if (nsteps < cap) t_out[nsteps] = zend;
    return FL_OK;
}

int fl_forward_evidence(fl_problem* pr, int nsave, double* ev_out) {
    Nvtx nvtx_("fl_forward_evidence");
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!ev_out || nsave < 1) return set_err(ctx, FL_EINVAL, "null argument");
    const int M = pr->m, nt = pr->nt;
    const double* d_save = nullptr;
    int status = FL_EINVAL;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    if (pr->use_mm) {
        MmWork* w = pr->mlast;
        if (w && w->B == 1 && w->nsave == nsave) {
            std::vector<MmState> st;
            rc = mm_read_states(ctx, w, 1, st);
            if (rc) return rc;
            status = st[0].phase == PH_DONE ? st[0].status : FL_EINVAL;
            d_save = w->d_save;
        }
    } else {
        Work* w = pr->last;
        if (w && w->B == 1 && w->nsave == nsave) {
            std::vector<SlotState> st;
            rc = read_states(ctx, w, st);
            if (rc) return rc;
            status = st[0].phase == PH_DONE ? st[0].status : FL_EINVAL;
            d_save = w->d_save;
        }
    }
    if (!d_save || status != FL_OK)
        return set_err(ctx, FL_EINVAL,
                       "fl_forward_evidence needs a completed fl_forward with %d save positions",
                       nsave);
    EvidenceFn fn = mm_evidence_launcher(ilog2i(nt));
    if (!fn) return set_err(ctx, FL_EUNSUPPORTED, "evidence for Nt = %d is not built", nt);
    const size_t bytes = sizeof(double) * (size_t)nsave * (kEvFixed + M);
    if (bytes > pr->ev_bytes) {
        CU(cudaStreamSynchronize(ctx->stream));
        cudaFree(pr->d_ev);
        pr->d_ev = nullptr;
        pr->ev_bytes = 0;
        CU(cudaMalloc(&pr->d_ev, bytes));
        pr->ev_bytes = bytes;
    }
    EvidenceArgs a{pr->d_tw[1], static_cast<const double*>(pr->d_ss[1]), d_save, nsave, M, nt,
                   pr->d_ev, ctx->stream};
    CU(fn(a));
    ctx->launches++;
    CU(cudaMemcpyAsync(ev_out, pr->d_ev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

int fl_rhs_eval(fl_problem* pr, int adjoint, double z, const double* u_in, const double* u_fwd,
                double* du_out) {
    Nvtx nvtx_("fl_rhs_eval");
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!u_in || !du_out || (adjoint && !u_fwd) || !std::isfinite(z))
        return set_err(ctx, FL_EINVAL, "invalid argument");
    if (adjoint && !pr->gamma_sym)
        return set_err(ctx, FL_NONSYMMETRIC,
                       "fiber adjoint requires a fully permutation-symmetric gamma tensor");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    if (pr->use_mm) return mm_rhs_eval(pr, adjoint, z, u_in, u_fwd, du_out);
    const int fp64 = pr->precision == FL_PRECISION_FP64;
    RhsFn fn = rhs_launcher(fp64, ilog2i(pr->nt));
    if (!fn) return set_err(ctx, FL_EUNSUPPORTED, "Nt = %d is not built", pr->nt);
    Work* w = nullptr;
    rc = new_work(pr, 1, 0, MODE_FORWARD, &w);
    if (rc) return rc;
    std::unique_ptr<Work> hold(w);
    const size_t bytes = 16 * (size_t)pr->nt * pr->m;
    CU(cudaMemcpyAsync(w->d_u0, u_in, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if (adjoint)
        CU(cudaMemcpyAsync(w->d_lamL, u_fwd, bytes, cudaMemcpyHostToDevice, ctx->stream));
    RhsArgs a{w->d_desc, adjoint, z, w->d_u0, adjoint ? w->d_lamL : nullptr, w->d_lam0,
              ctx->stream};
    CU(fn(a));
    ctx->launches++;
    CU(cudaMemcpyAsync(du_out, w->d_lam0, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

static int phase_gradient_core(fl_problem* pr, Work* w, int nbatch, const double* d_u0,
                               const double* d_phases, const unsigned char* d_mask,
                               int log_cost, double* d_J, double* d_grad, fl_stats* stats) {
    Nvtx nvtx_("fl: batched forward + adjoint + gradient");
    fl_ctx* ctx = pr->ctx;
    const int nt = pr->nt;
    CU(cudaEventRecord(ctx->ev[0], ctx->stream));
    int rc = set_mode(ctx, w, MODE_BAND_GRADIENT, log_cost, pr->objective, pr->obj_tau);
    if (rc) return rc;
    CU(cudaMemsetAsync(w->d_state, 0, sizeof(SlotState) * nbatch, ctx->stream));
    CU(cudaMemcpyAsync(w->d_mask, d_mask, nt, cudaMemcpyDeviceToDevice, ctx->stream));
    const int threads = 256;
    const long total = (long)nt * nbatch;
    const int blocks = (int)std::min<long>((total + threads - 1) / threads, 4096);
    shaped_launch_kernel<<<blocks, threads, 0, ctx->stream>>>(
        (const double2*)d_u0, d_phases, nt, 1, nbatch, (double2*)w->d_u0, (size_t)nt);
    ctx->launches++;
    CU(cudaGetLastError());
    rc = run_to_completion(pr, w);
    if (rc) return rc;
    gather_stats_kernel<<<(nbatch + 255) / 256, 256, 0, ctx->stream>>>(w->d_state, nbatch, d_J);
    ctx->launches++;
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(d_grad, w->d_grad, 8 * (size_t)nt * nbatch, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    CU(cudaEventRecord(ctx->ev[1], ctx->stream));
    std::vector<SlotState> st;
    rc = read_states(ctx, w, st);
    if (rc) return rc;
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->call_ms = ms;
    if (stats)
        for (int b = 0; b < nbatch; b++) fill_stats(st[b], &stats[b]);
    return status_of_slots(ctx, st);
}

static int phase_gradient_device(fl_problem* pr, const double* d_u0, int nbatch,
                                 const double* d_phases, int per_mode,
                                 const unsigned char* d_mask, int log_cost, double* d_J,
                                 double* d_grad, fl_stats* stats) {
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!d_u0 || !d_phases || !d_mask || !d_J || !d_grad || nbatch < 1)
        return set_err(ctx, FL_EINVAL, "null argument");
    if (!pr->gamma_sym)
        return set_err(ctx, FL_NONSYMMETRIC,
                       "fiber adjoint requires a fully permutation-symmetric gamma tensor");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    if (pr->use_mm)
        return mm_phase_gradient_device(pr, d_u0, nbatch, d_phases, per_mode && pr->m > 1, d_mask,
                                        log_cost, d_J, d_grad, stats);
    // single mode: a per-mode phase is the shared phase
    // keep one workspace per problem sized for the largest batch seen
    if (!pr->last || pr->last->B < nbatch || pr->last->nsave != 0) {
        delete pr->last;
        pr->last = nullptr;
        Work* w = nullptr;
        rc = new_work(pr, nbatch, 0, MODE_BAND_GRADIENT, &w);
        if (rc) return rc;
        pr->last = w;
    }
    Work* w = pr->last;
    const int B = w->B;
    if (B != nbatch) {
        // run only the first nbatch slots
        w->B = nbatch;
        rc = phase_gradient_core(pr, w, nbatch, d_u0, d_phases, d_mask, log_cost, d_J, d_grad,
                                 stats);
        w->B = B;
        return rc;
    }
    return phase_gradient_core(pr, w, nbatch, d_u0, d_phases, d_mask, log_cost, d_J, d_grad,
                               stats);
}

// host-buffer form: copies in, runs the device form, copies out
static int phase_gradient_host(fl_problem* pr, const double* u0, int nbatch,
                               const double* phases, int per_mode, const unsigned char* mask,
                               int log_cost, double* J, double* grad, fl_stats* stats) {
    int rc = check_problem(pr);
    if (rc) return rc;
    fl_ctx* ctx = pr->ctx;
    if (!u0 || !phases || !mask || !J || !grad || nbatch < 1)
        return set_err(ctx, FL_EINVAL, "null argument");
    const int nt = pr->nt;
    const size_t nm = (size_t)nt * pr->m;
    const size_t np = (per_mode ? nm : (size_t)nt) * nbatch;  // phase (and gradient) values
    bool any = false;
    for (int i = 0; i < nt; i++) any |= mask[i] != 0;
    if (!any) return set_err(ctx, FL_EINVAL, "band mask must contain at least one bin");
    // every phase must be finite: a large batch is scanned on a host thread
    // while the GPU runs it (the scan reads the whole input once, several ms
    // at 592 x 2^13 values); a call with a non-finite phase still returns
    // FL_EINVAL and writes no output
    auto nonfinite = [phases](size_t lo, size_t hi) {
        uint64_t bad = 0;
        for (size_t i = lo; i < hi; i++) {
            uint64_t b;
            memcpy(&b, &phases[i], 8);
            bad |= (uint64_t)(((b >> 52) & 0x7ff) == 0x7ff);
        }
        return bad != 0;
    };
    bool bad_phase = false;
    std::thread scan;
    if (np < ((size_t)1 << 20)) {
        if (nonfinite(0, np)) return set_err(ctx, FL_EINVAL, "phase values must be finite");
    } else {
        scan = std::thread([&] { bad_phase = nonfinite(0, np); });
    }
    struct Join {
        std::thread& t;
        ~Join() {
            if (t.joinable()) t.join();
        }
    } join_scan{scan};
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, FL_ENODEV, "cudaSetDevice");
    // inputs and outputs in the problem's staging area: one allocation that
    // grows to the largest batch seen and is reused by later calls
    auto up256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t need = up256(16 * nm) + 2 * up256(8 * np) + up256(8 * (size_t)nbatch) + up256(nt);
    if (need > pr->stage_bytes) {
        CU(cudaStreamSynchronize(ctx->stream));
        cudaFree(pr->d_stage);
        pr->d_stage = nullptr;
        pr->stage_bytes = 0;
        CU(cudaMalloc(&pr->d_stage, need));
        pr->stage_bytes = need;
    }
    char* sp = pr->d_stage;
    double* d_u0 = reinterpret_cast<double*>(sp);
    sp += up256(16 * nm);
    double* d_ph = reinterpret_cast<double*>(sp);
    sp += up256(8 * np);
    double* d_g = reinterpret_cast<double*>(sp);
    sp += up256(8 * np);
    double* d_J = reinterpret_cast<double*>(sp);
    sp += up256(8 * (size_t)nbatch);
    unsigned char* d_m = reinterpret_cast<unsigned char*>(sp);
    CU(cudaMemcpyAsync(d_u0, u0, 16 * nm, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(d_ph, phases, 8 * np, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(d_m, mask, nt, cudaMemcpyHostToDevice, ctx->stream));
    rc = phase_gradient_device(pr, d_u0, nbatch, d_ph, per_mode, d_m, log_cost, d_J, d_g, stats);
    if (scan.joinable()) scan.join();
    if (bad_phase) {
        CU(cudaStreamSynchronize(ctx->stream));
        return set_err(ctx, FL_EINVAL, "phase values must be finite");
    }
    if (rc == FL_OK) {
        CU(cudaMemcpyAsync(J, d_J, 8 * (size_t)nbatch, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(grad, d_g, 8 * np, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    return rc;
}

int fl_phase_gradient_batch_device(fl_problem* pr, const double* d_u0, int nbatch,
                                   const double* d_phases, const unsigned char* d_mask,
                                   int log_cost, double* d_J, double* d_grad, fl_stats* stats) {
    return phase_gradient_device(pr, d_u0, nbatch, d_phases, 0, d_mask, log_cost, d_J, d_grad,
                                 stats);
}

int fl_phase_gradient_batch(fl_problem* pr, const double* u0, int nbatch, const double* phases,
                            const unsigned char* mask, int log_cost, double* J, double* grad,
                            fl_stats* stats) {
    return phase_gradient_host(pr, u0, nbatch, phases, 0, mask, log_cost, J, grad, stats);
}

int fl_mode_phase_gradient_batch_device(fl_problem* pr, const double* d_u0, int nbatch,
                                        const double* d_phases, const unsigned char* d_mask,
                                        int log_cost, double* d_J, double* d_grad,
                                        fl_stats* stats) {
    if (pr && pr->m == 1)
        return phase_gradient_device(pr, d_u0, nbatch, d_phases, 0, d_mask, log_cost, d_J,
                                     d_grad, stats);
    return phase_gradient_device(pr, d_u0, nbatch, d_phases, 1, d_mask, log_cost, d_J, d_grad,
                                 stats);
}

int fl_mode_phase_gradient_batch(fl_problem* pr, const double* u0, int nbatch,
                                 const double* phases, const unsigned char* mask, int log_cost,
                                 double* J, double* grad, fl_stats* stats) {
    return phase_gradient_host(pr, u0, nbatch, phases, pr && pr->m > 1 ? 1 : 0, mask, log_cost,
                               J, grad, stats);
}

int fl_server_create(fl_ctx* ctx, const fl_server_opts* opts, fl_server** out) {
    if (!ctx || !out) return FL_EINVAL;
    *out = nullptr;
    auto sv = std::make_unique<fl_server>();
    sv->ctx = ctx;
    sv->opts.hbm_budget_bytes = (size_t)120 << 30;
    sv->opts.evals_per_launch = 48;
    sv->opts.checkpoints = 256;
    sv->opts.segment_steps = 128;
    if (opts) {
        if (opts->hbm_budget_bytes) sv->opts.hbm_budget_bytes = opts->hbm_budget_bytes;
        if (opts->evals_per_launch > 0) sv->opts.evals_per_launch = opts->evals_per_launch;
        if (opts->checkpoints > 0) sv->opts.checkpoints = opts->checkpoints;
        if (opts->segment_steps > 0) sv->opts.segment_steps = opts->segment_steps;
    }
    // default: no cap beyond slots and memory (a cap at the SM count trades
    // median latency for nothing on a heavy-tailed stream)
    sv->opts.max_active_ctas =
        opts && opts->max_active_ctas > 0 ? opts->max_active_ctas : 1 << 30;
    if (!pow2(sv->opts.checkpoints) || sv->opts.checkpoints < 2)
        return set_err(ctx, FL_EINVAL, "server checkpoints must be a power of two >= 2");
    sv->wopts = ctx->opts;
    sv->wopts.checkpoints = sv->opts.checkpoints;
    sv->wopts.segment_steps = sv->opts.segment_steps;
    sv->wopts.step_log = 0;  // one entry per allowed attempted step
    sv->wopts.max_iters = std::max(ctx->opts.max_iters, 400000L);
    fl_server* p = sv.release();
    p->th = std::thread(srv_thread, p);
    *out = p;
    return FL_OK;
}

int fl_server_destroy(fl_server* sv) {
    if (!sv) return FL_EINVAL;
    sv->stop.store(true);
    if (sv->th.joinable()) sv->th.join();
    cudaSetDevice(sv->ctx->device);
    for (auto* b : sv->buckets) {
        for (auto* c : b->chunks)
            if (c->stream) cudaStreamSynchronize(c->stream);
        delete b;
    }
    // every request not yet handed back is in reqs (queued, running or finished)
    for (auto& kv : sv->reqs) delete kv.second;
    delete sv;
    return FL_OK;
}

int fl_server_submit(fl_server* sv, const fl_request* q, long* id) {
    if (!sv || !q || !id || !q->prob || !q->u0) return FL_EINVAL;
    fl_ctx* ctx = sv->ctx;
    fl_problem* pr = q->prob;
    if (q->kind != FL_REQ_FORWARD && q->kind != FL_REQ_BAND_GRADIENT)
        return set_err(ctx, FL_EINVAL, "unknown request kind %d", q->kind);
    if (q->kind == FL_REQ_BAND_GRADIENT) {
        if (!q->phase || !q->mask || !q->out_grad)
            return set_err(ctx, FL_EINVAL, "band-gradient request needs phase, mask and out_grad");
        if (!pr->gamma_sym)
            return set_err(ctx, FL_NONSYMMETRIC,
                           "fiber adjoint requires a fully permutation-symmetric gamma tensor");
    } else if (!q->out_field) {
        return set_err(ctx, FL_EINVAL, "forward request needs out_field");
    }
    const int logn = ilog2i(pr->nt);
    if (pr->use_mm ? !mm_round_launcher(logn)
                   : !sm_launcher(pr->precision == FL_PRECISION_FP64, logn))
        return set_err(ctx, FL_EUNSUPPORTED, "shape not built (Nt = %d, M = %d)", pr->nt, pr->m);
    const size_t one = srv_slot_bytes(sv, pr) * 1;
    if (sv->opts.hbm_budget_bytes && one > sv->opts.hbm_budget_bytes)
        return set_err(ctx, FL_OOM_ADMISSION, "one slot of %zu bytes exceeds the HBM budget", one);
    const double L = q->L > 0 ? q->L : pr->L;
    if (!std::isfinite(L)) return set_err(ctx, FL_EINVAL, "L must be positive and finite");
    auto r = std::make_unique<SrvRequest>();
    r->prob = pr;
    r->weight = pr->use_mm ? pr->m * mm_cluster_ctas(logn) : 1;
    r->kind = q->kind;
    r->log_cost = q->log_cost;
    r->objective = pr->objective;
    r->obj_tau = pr->obj_tau;
    r->L = L;
    const size_t nm = (size_t)pr->nt * pr->m;
    r->u0.assign(q->u0, q->u0 + 2 * nm);
    double nrm = 0.0;
    for (double x : r->u0) {
        if (!std::isfinite(x)) return set_err(ctx, FL_EINVAL, "input spectrum must be finite");
        nrm += x * x;
    }
    if (!(nrm > 0)) return set_err(ctx, FL_EINVAL, "input spectrum must be nonzero");
    if (q->kind == FL_REQ_BAND_GRADIENT) {
        bool any = false;
        r->mask.assign(q->mask, q->mask + pr->nt);
        for (auto x : r->mask) any |= x != 0;
        if (!any) return set_err(ctx, FL_EINVAL, "band mask must contain at least one bin");
        // u_shaped = u0 ⊙ cis(φ) (physics_models.jl:791-797)
        for (size_t k = 0; k < nm; k++) {
            const double ph = q->phase[k % pr->nt];
            if (!std::isfinite(ph)) return set_err(ctx, FL_EINVAL, "phase values must be finite");
            const double c = std::cos(ph), s = std::sin(ph), a = r->u0[2 * k], b = r->u0[2 * k + 1];
            r->u0[2 * k] = a * c - b * s;
            r->u0[2 * k + 1] = a * s + b * c;
        }
        r->out_grad = q->out_grad;
    } else {
        r->out_field = q->out_field;
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->fatal) return set_err(ctx, sv->fatal, "server stopped: %s", sv->err.c_str());
    r->id = sv->next_id++;
    r->t_submit = now_ms();
    *id = r->id;
    sv->reqs[r->id] = r.get();
    sv->incoming.push_back(r.release());
    sv->submitted++;
    return FL_OK;
}

static int srv_result(fl_server* sv, SrvRequest* r, fl_stats* stats, double* J, double* lat) {
    if (stats) *stats = r->stats;
    if (J) *J = r->J;
    if (lat) *lat = r->t_done - r->t_submit;
    const int st = r->status;
    sv->reqs.erase(r->id);
    delete r;
    return st;
}

int fl_server_poll(fl_server* sv, long id, fl_stats* stats, double* J, double* latency_ms) {
    if (!sv) return FL_EINVAL;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return FL_EINVAL;
    if (it->second->status == FL_EBUSY) return FL_EBUSY;
    return srv_result(sv, it->second, stats, J, latency_ms);
}

int fl_server_wait(fl_server* sv, long id, double timeout_ms, fl_stats* stats, double* J,
                   double* latency_ms) {
    if (!sv) return FL_EINVAL;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return FL_EINVAL;
    SrvRequest* r = it->second;
    const auto until = std::chrono::steady_clock::now() +
                       std::chrono::microseconds((long)(std::max(0.0, timeout_ms) * 1000));
    while (r->status == FL_EBUSY)
        if (sv->cv.wait_until(lk, until) == std::cv_status::timeout && r->status == FL_EBUSY)
            return FL_TIMEOUT;
    return srv_result(sv, r, stats, J, latency_ms);
}

int fl_server_info_get(fl_server* sv, fl_server_info* info) {
    if (!sv || !info) return FL_EINVAL;
    std::lock_guard<std::mutex> lk(sv->mu);
    info->submitted = sv->submitted;
    info->completed = sv->completed;
    info->queued = (long)sv->incoming.size() + sv->n_waiting.load();
    info->in_flight = sv->submitted - sv->completed;
    int slots = 0, chunks = 0;
    for (auto* b : sv->buckets) {
        chunks += (int)b->chunks.size();
        for (auto* c : b->chunks) slots += c->B;
    }
    info->slots = slots;
    info->chunks = chunks;
    info->hbm_bytes = sv->hbm_used;
    info->launches = sv->launches;
    return FL_OK;
}

}  // extern "C"
