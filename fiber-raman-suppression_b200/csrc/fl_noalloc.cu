// fl_noalloc.cu -- forward solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc: host runtimes whose device memory is
// owned by their own pool allocator (a Julia or Python process that has
// reserved the device up front), or a latency-critical request loop that
// must not hit cudaMalloc's implicit device synchronisation.  This entry
// point runs the single-mode forward stepper on device buffers the caller
// already owns and keeps everything else -- the slot descriptor, the solver
// state, the derived spectral tables and the stepper's workspace -- in one
// file-scope device array of fixed size.  That array exists once per GPU
// that loads the library and stays resident until the process exits.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>

#include "../../include/fiberlab_gpu.h"
#include "fl_launch.h"

using namespace fl;

namespace {

// Scratch budget: descriptor, state and tables plus the FP32 forward
// workspace (two FP64 states, seven FP32 stages, scratch fields, the error
// buffers).  A forward-only solve keeps no step log and no checkpoints, so
// the number of steps is not limited by the scratch size.
constexpr size_t kScratchBytes = 2u << 20;  // 2 MiB per device
constexpr int kMaxLogN = 13;                // Nt <= 2^13
constexpr int kMinLogN = 6;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {nullptr};  // device address of g_scratch, per device

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Offsets of every region inside the scratch array for nt points.
struct Layout {
    size_t desc, state, active, dturns, heff, ss, tw, u0b, u1b, kf[7], scr0, scr1, esv, skv, end;
    explicit Layout(int nt) {
        size_t p = 0;
        auto take = [&](size_t bytes) {
            size_t r = p;
            p = align256(p + bytes);
            return r;
        };
        desc = take(sizeof(SlotDesc));
        state = take(sizeof(SlotState));
        active = take(sizeof(int));
        dturns = take(8 * (size_t)nt);
        heff = take(8 * (size_t)nt);
        ss = take(4 * (size_t)nt);
        tw = take(8 * (size_t)nt);
        u0b = take(16 * (size_t)nt);
        u1b = take(16 * (size_t)nt);
        for (int i = 0; i < 7; i++) kf[i] = take(8 * (size_t)nt);
        scr0 = take(16 * (size_t)nt);
        scr1 = take(16 * (size_t)nt);
        esv = take(16 * (size_t)nt);
        skv = take(8 * (size_t)nt);
        end = p;
    }
};

// Builds the derived tables and the slot descriptor inside the scratch,
// zeroes the solver state and checks the caller's save positions and launch
// (a failed check leaves the slot finished with FL_EINVAL).
__global__ void noalloc_prepare(SlotDesc desc, unsigned char* base, Layout lay, int nt,
                                const double* __restrict__ D, const double* __restrict__ hR,
                                const double* __restrict__ selfsteep) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nt) {
        reinterpret_cast<double*>(base + lay.dturns)[i] = D[i] / (2.0 * M_PI);
        const double sg = (i & 1) ? -1.0 : 1.0;  // fftshift folded into the response
        reinterpret_cast<float2*>(base + lay.heff)[i] =
            make_float2((float)(hR[2 * i] * sg), (float)(hR[2 * i + 1] * sg));
        reinterpret_cast<float*>(base + lay.ss)[i] = (float)selfsteep[i];
        double s, c;
        sincospi(-2.0 * (double)i / (double)nt, &s, &c);
        reinterpret_cast<float2*>(base + lay.tw)[i] = make_float2((float)c, (float)s);
    }
    if (i == 0) {
        *reinterpret_cast<SlotDesc*>(base + lay.desc) = desc;
        SlotState* st = reinterpret_cast<SlotState*>(base + lay.state);
        *st = SlotState{};  // the state must start at zero (phase = first step)
        *reinterpret_cast<int*>(base + lay.active) = 0;
        bool ok = desc.nsave >= 2 && desc.zsave[0] == 0.0 && desc.zsave[desc.nsave - 1] == desc.L;
        for (int k = 1; ok && k < desc.nsave; k++)
            ok = isfinite(desc.zsave[k]) && desc.zsave[k] > desc.zsave[k - 1];
        double nrm = 0.0;
        for (int k = 0; ok && k < 2 * nt; k++) {
            ok = isfinite(desc.u0[k]);
            nrm += desc.u0[k] * desc.u0[k];
        }
        if (!ok || !(nrm > 0)) {
            st->status = FL_EINVAL;
            st->phase = PH_DONE;
        }
    }
}

// Restores the calling thread's current device on every return path: the
// callers of this entry point (host runtimes that own the device) must not
// find their thread moved to another device.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) return;
        ok = prev == device || cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (ok && prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int fl_forward_noalloc(int device, int nt, const double* d_D, double gamma,
                                  const double* d_hR, const double* d_selfsteep,
                                  double one_m_fR, double L, double reltol, double abstol,
                                  const double* d_u0, const double* d_saveat, int nsave,
                                  double* d_out_spectra, void* stream, fl_stats* stats) {
    int logn = 0;
    while ((1 << logn) < nt) logn++;
    if (nt < 1 || (1 << logn) != nt || logn < kMinLogN || logn > kMaxLogN) return FL_EUNSUPPORTED;
    if (!d_D || !d_hR || !d_selfsteep || !d_u0 || !d_saveat || !d_out_spectra || nsave < 2)
        return FL_EINVAL;
    if (!(std::isfinite(L) && L > 0) || !(std::isfinite(reltol) && reltol > 0) ||
        !(std::isfinite(abstol) && abstol > 0) || !std::isfinite(gamma) ||
        !std::isfinite(one_m_fR))
        return FL_EINVAL;
    if (device < 0 || device >= kMaxDevices) return FL_ENODEV;
    const Layout lay(nt);
    if (lay.end > kScratchBytes) return FL_EUNSUPPORTED;
    DeviceGuard guard(device);
    if (!guard.ok) return FL_ENODEV;
    // an error left pending by earlier work on this thread is not this
    // call's: report it without consuming it
    if (cudaPeekAtLastError() != cudaSuccess) return FL_ECUDA;
    // one-time set-up per device (with that device current): the device
    // address of the scratch array; the host-side symbol is not a device address
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return FL_ECUDA;
        g_scratch_addr[device] = p;
    }
    unsigned char* base = static_cast<unsigned char*>(g_scratch_addr[device]);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    SlotDesc d{};
    d.Dturns = reinterpret_cast<const double*>(base + lay.dturns);
    d.Heff[0] = base + lay.heff;
    d.ss[0] = base + lay.ss;
    d.tw[0] = base + lay.tw;
    d.gamma = gamma;
    d.one_m_fR = one_m_fR;
    d.L = L;
    d.reltol = reltol;
    d.abstol = abstol;
    d.mode = MODE_FORWARD;
    d.nsave = nsave;
    d.ck_cap = 0;    // forward only: no z-checkpoints,
    d.seg_cap = 0;
    d.step_cap = 0;  // no step log (nothing is kept for an adjoint)
    d.max_iters = 100000;
    d.zsave = d_saveat;
    d.save_out = d_out_spectra;
    d.u0 = d_u0;
    d.u[0] = reinterpret_cast<double*>(base + lay.u0b);
    d.u[1] = reinterpret_cast<double*>(base + lay.u1b);
    for (int i = 0; i < 7; i++) d.kf[i] = base + lay.kf[i];
    d.scr[0] = base + lay.scr0;
    d.scr[1] = base + lay.scr1;
    d.esv = reinterpret_cast<double*>(base + lay.esv);
    d.skv = reinterpret_cast<double*>(base + lay.skv);

    noalloc_prepare<<<(nt + 255) / 256, 256, 0, s>>>(d, base, lay, nt, d_D, d_hR, d_selfsteep);
    if (cudaGetLastError() != cudaSuccess) return FL_ECUDA;  // this launch's own error
    LaunchFn fn = sm_launcher(0, logn);
    if (!fn) return FL_EUNSUPPORTED;
    LaunchArgs a{base + lay.desc, reinterpret_cast<SlotState*>(base + lay.state),
                 reinterpret_cast<const int*>(base + lay.active), 1, INT_MAX, s};
    if (fn(a) != cudaSuccess) return FL_ECUDA;
    SlotState st;
    if (cudaMemcpyAsync(&st, base + lay.state, sizeof st, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return FL_ECUDA;
    if (stats) {
        stats->naccept = st.naccept;
        stats->nreject = st.nreject;
        stats->nf = st.nf;
        stats->adj_naccept = stats->adj_nreject = stats->adj_nf = 0;
        stats->status = st.status;
        stats->checkpoints_used = 0;
        stats->J = 0.0;
        stats->z_end = st.z;
        stats->recompute_steps = 0;
    }
    return st.status;
}
