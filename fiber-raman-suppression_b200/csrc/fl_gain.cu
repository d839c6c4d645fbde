// fl_gain.cu -- pump-gain single-mode forward stepper (disp_gain_smf!).
//
// Reference: the right-hand side src/simulation/simulate_disp_gain_mmf.jl:
// 21-66 (disp_mmf!'s nonlinear term plus g(ω)ũ/2, and dP/dz = g_P P), the
// gain models :68-102 with calculate_gain_YDFA (src/gain_simulation/gain.jl:
// 150-166), and the solver :204-239 (Tsit5 over the state [P; ũ]).
//
// One CTA integrates one problem to z = L in one launch.  The nonlinear term
// is the single-mode stepper's forward right-hand side (its transforms, with
// the field handed over through the shared transform buffer).  The gain of a
// stage is computed from the stage input before that call: two block sums
// give the rate-equation terms W12 and W21 of the stage's spectrum (|ũ|² =
// |e^{iDz}ũ|²), the inversion n2 follows, and each thread keeps g_b ũ_b / 2
// of its own bins in scratch and adds it to the returned derivative.  The
// pump power and its seven stage derivatives are block-uniform FP64 scalars;
// the RMS error norm runs over the Nt + 1 components of the state, as the
// reference's does over [P; ũ].  FP32 right-hand side, FP64 state, stage
// accumulation and error norm, as the main stepper.
#include "fl_launch.h"
#include "fl_sm.cuh"

namespace fl {

template <int LOGN, int LOGE>
__global__ void __launch_bounds__(FftShape<LOGN, LOGE>::T, 1)
    gain_forward_kernel(const GainDesc* __restrict__ gdp, GainOut* __restrict__ out) {
    using Sol = SmSolver<float, LOGN, LOGE>;
    using CF = cx<float>;
    using IO = FieldIO<CF, LOGN, LOGE>;
    static_assert(IO::SMEM, "the stage field is handed over in shared memory");
    constexpr int N = Sol::N, E = Sol::E, T = Sol::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* red = reinterpret_cast<double*>(smraw + SmemPlan<double, LOGN>::BYTES);
    const GainDesc& g = *gdp;
    const SlotDesc& d = g.s;
    load_twiddles<LOGN>(d, red);
    Sol S(d, smraw, red);
    const IO io{reinterpret_cast<CF*>(smraw)};
    CF* gb = static_cast<CF*>(d.scr[1]);  // g_b ũ_b / 2 of the current stage
    CF* k[7];
#pragma unroll
    for (int i = 0; i < 7; i++) k[i] = static_cast<CF*>(d.kf[i]);
    double* u = d.u[0];
    double* un = d.u[1];
    const double L = d.L, dtmin = kEps * L, at = d.abstol, rt = d.reltol;

    // g(ω)ũ/2 of the stage in io into gb (own bins); returns g_P
    auto gain_of_stage = [&](double pp) -> double {
        if (g.kind == 0) {
#pragma unroll
            for (int s = 0; s < E; s++) gb[Sol::bin(s)] = scale(io[s], (float)(0.5 * g.g_const));
            return -1.0;
        }
        double w12 = 0.0, w21 = 0.0;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = Sol::bin(s);
            const double e = abs2(up(io[s]));
            w12 += g.wa[b] * e;
            w21 += g.we[b] * e;
        }
        w12 = block_sum<T>(w12, red);
        w21 = block_sum<T>(w21, red);
        const double r12 = g.r12c * pp, r21 = g.r21c * pp;
        const double n2 = (r12 + w12) / (r12 + r21 + w12 + w21 + g.inv_tau), n1 = 1.0 - n2;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = Sol::bin(s);
            gb[b] = scale(io[s], (float)(0.5 * (g.sE[b] * n2 - g.sA[b] * n1)));
        }
        return g.gpe * n2 - g.gpa * n1;
    };
    // derivative of the stage (field in io, pump pp) at z: io <- dũ, returns dP
    auto deriv = [&](double z, double pp) -> double {
        const double gP = gain_of_stage(pp);
        rhs_fwd_call<float, LOGN, LOGE>(&d, smraw, red, z, io);
#pragma unroll
        for (int s = 0; s < E; s++) io[s] = io[s] + gb[Sol::bin(s)];
        return gP * pp;
    };

    // ---- launch and f0
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = Sol::bin(s);
        const cx<double> x = ld2(d.u0, b);
        st2(u, b, x);
        io[s] = down<float>(x);
    }
    double pp = g.pump0;
    // save positions at z = 0: the launch (the lab frame equals the interaction frame there)
    int save_idx = 0;
    while (save_idx < d.nsave && d.zsave[save_idx] == 0.0) {
        double* o = d.save_out + (size_t)save_idx * 2 * N;
#pragma unroll
        for (int s = 0; s < E; s++) st2(o, Sol::bin(s), ld2(d.u0, Sol::bin(s)));
        if (threadIdx.x == 0) g.pump_save[save_idx] = pp;
        save_idx++;
    }
    long nf = 0, naccept = 0, nreject = 0;
    int status = ST_OK;
    double kp[7];
    kp[0] = deriv(0.0, pp);
    nf++;
#pragma unroll
    for (int s = 0; s < E; s++) k[0][Sol::bin(s)] = io[s];

    // ---- initial step (OrdinaryDiffEqCore ode_determine_initdt), P one more
    // component of the norms; weights from the launch
    const double skp = at + fabs(pp) * rt;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = Sol::bin(s);
        const cx<double> x = ld2(u, b);
        const double ax = sqrt(x.re * x.re + x.im * x.im), sk = at + ax * rt;
        const double af = sqrt(abs2(up(io[s])));
        s0 += (ax / sk) * (ax / sk);
        s1 += (af / sk) * (af / sk);
    }
    s0 = block_sum<T>(s0, red) + (pp / skp) * (pp / skp);
    s1 = block_sum<T>(s1, red) + (kp[0] / skp) * (kp[0] / skp);
    const double d0 = sqrt(s0 / (N + 1)), d1 = sqrt(s1 / (N + 1));
    double dt;
    if (isnan(d1)) {
        dt = dtmin;
    } else {
        const double dt0 = fmin((d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : (d0 / d1) / 100.0, L);
        if (dt0 < 10.0 * kEps) {
            dt = fmax(1e-6, dtmin);
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int b = Sol::bin(s);
                const cx<double> x = ld2(u, b);
                const CF f0 = k[0][b];
                io[s] = mk((float)(x.re + dt0 * (double)f0.re), (float)(x.im + dt0 * (double)f0.im));
            }
            const double kp1 = deriv(dt0, pp + dt0 * kp[0]);
            nf++;
            double s2 = 0.0, nd = 0.0;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int b = Sol::bin(s);
                const cx<double> x = ld2(u, b);
                const double sk = at + sqrt(x.re * x.re + x.im * x.im) * rt;
                const CF f0 = k[0][b];
                const double dr = (double)io[s].re - (double)f0.re;
                const double di = (double)io[s].im - (double)f0.im;
                s2 += (dr * dr + di * di) / (sk * sk);
                nd += (dr != 0.0 || di != 0.0) ? 1.0 : 0.0;
            }
            const double dp = kp1 - kp[0];
            s2 = block_sum<T>(s2, red) + (dp / skp) * (dp / skp);
            nd = block_sum<T>(nd, red) + (dp != 0.0 ? 1.0 : 0.0);
            const double d2 = sqrt(s2 / (N + 1)) / dt0;
            dt = initdt_final(dt0, d1, d2, nd, dtmin, L);
        }
    }
    nf++;  // the reference evaluates f0 once more after the initial step

    // ---- Tsit5 with the PI controller, FSAL (k0 <- k6 on accept)
    double z = 0.0, qold = kQoldInit;
    long iters = 0;
    while (z < L) {
        if (++iters > d.max_iters) {
            status = ST_MAXITERS;
            break;
        }
        double adt = fmax(fmin(fabs(dt), L), dtmin);
        const double rem = L - z;
        if (adt > rem) adt = rem;
        if (adt <= dtmin && rem > dtmin) {
            status = ST_DT_UNDERFLOW;
            break;
        }
        dt = adt;
        double pnew = pp;
        for (int st = 1; st < 7; st++) {
            double acc = 0.0;
            for (int j = 0; j < st; j++) acc += kT5a[st][j] * kp[j];
            const double pps = pp + dt * acc;
            if (st < 6) {
                S.stage_input(st, u, d.kf, 0, dt, io);
            } else {
                S.stage7_input(u, un, d.kf, 0, dt, at, rt, io, true);
                pnew = pps;
            }
            kp[st] = deriv(z + kT5c[st] * dt, pps);
            nf++;
#pragma unroll
            for (int s = 0; s < E; s++) k[st][Sol::bin(s)] = io[s];
        }
        // error dt Σ b̃_j k_j over the Nt + 1 components
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = Sol::bin(s);
            const cx<double> e6 = ld2(d.esv, b);
            const double er = e6.re + dt * kT5bt[6] * (double)io[s].re;
            const double ei = e6.im + dt * kT5bt[6] * (double)io[s].im;
            const double w = d.skv[b];
            acc += (er * er + ei * ei) / (w * w);
        }
        acc = block_sum<T>(acc, red);
        double ep = 0.0;
        for (int j = 0; j < 7; j++) ep += kT5bt[j] * kp[j];
        ep *= dt;
        const double wp = at + fmax(fabs(pp), fabs(pnew)) * rt;
        const double EEst = sqrt((acc + (ep / wp) * (ep / wp)) / (N + 1));
        if (!isfinite(EEst)) {
            status = ST_NONFINITE;
            break;
        }
        double q11;
        const double q = pi_q(EEst, qold, q11);
        if (EEst > 1.0) {
            nreject++;
            dt = dt / fmin(1.0 / kQmin, q11 / kGamma);
            continue;
        }
        naccept++;
        double znew = z + dt;
        if (fabs(znew - L) < 100.0 * kEps * fmax(z, L)) znew = L;  // snap to the tstop
        // save positions in (z, znew) and on an interior step end: Tsit5's
        // free interpolant u_n + dt Σ_i b_i(θ) k_i for the field and the pump
        // power (positions at L take the final state below)
        while (save_idx < d.nsave && d.zsave[save_idx] > z &&
               (d.zsave[save_idx] < znew || (d.zsave[save_idx] == znew && znew < L))) {
            const double zs = d.zsave[save_idx], th = (zs - z) / dt;
            double bi[7];
            for (int i = 0; i < 7; i++) {
                double b = 0.0, tp = th;
                for (int q = 0; q < 4; q++) {
                    b += kT5r[i][q] * tp;
                    tp *= th;
                }
                bi[i] = b;
            }
            double* o = d.save_out + (size_t)save_idx * 2 * N;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int b = Sol::bin(s);
                double xr = 0.0, xi = 0.0;
                for (int i = 0; i < 7; i++) {
                    const CF ki = k[i][b];
                    xr += bi[i] * (double)ki.re;
                    xi += bi[i] * (double)ki.im;
                }
                const cx<double> un0 = ld2(u, b);
                const cx<double> x = mk(un0.re + dt * xr, un0.im + dt * xi);
                const cx<double> p = phasor<double>(d.Dturns[b], zs);
                st2(o, b, mk(x.re * p.re - x.im * p.im, x.re * p.im + x.im * p.re));
            }
            if (threadIdx.x == 0) {
                double pk = 0.0;
                for (int i = 0; i < 7; i++) pk += bi[i] * kp[i];
                g.pump_save[save_idx] = pp + dt * pk;
            }
            save_idx++;
        }
        z = znew;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = Sol::bin(s);
            st2(u, b, ld2(un, b));
            k[0][b] = io[s];
        }
        pp = pnew;
        kp[0] = kp[6];
        qold = fmax(EEst, kQoldInit);
        dt = fmin(fmax((q == 1.0) ? dt : dt / q, dtmin), L);
    }

    // ---- lab-frame spectrum at the end (and the save positions at L), pump
    // power and counters
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = Sol::bin(s);
        const cx<double> x = ld2(u, b);
        const cx<double> p = phasor<double>(d.Dturns[b], z);
        const cx<double> y = mk(x.re * p.re - x.im * p.im, x.re * p.im + x.im * p.re);
        st2(d.uL_out, b, y);
        if (status == ST_OK)
            for (int si = save_idx; si < d.nsave; si++) st2(d.save_out + (size_t)si * 2 * N, b, y);
    }
    if (threadIdx.x == 0 && status == ST_OK)
        for (int si = save_idx; si < d.nsave; si++) g.pump_save[si] = pp;
    if (threadIdx.x == 0) {
        out->naccept = naccept;
        out->nreject = nreject;
        out->nf = nf;
        out->status = status;
        out->z_end = z;
        out->pump_L = pp;
    }
}

template <int LOGN, int LOGE>
cudaError_t launch_gain_t(const GainDesc* desc, GainOut* out, cudaStream_t stream) {
    auto kern = gain_forward_kernel<LOGN, LOGE>;
    const size_t smem = smem_bytes<double, LOGN>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<1, FftShape<LOGN, LOGE>::T, smem, stream>>>(desc, out);
    return cudaGetLastError();
}

bool gain_built(int logn) { return logn >= 6 && logn <= 13; }

cudaError_t launch_gain(int logn, const GainDesc* desc, GainOut* out, cudaStream_t stream) {
    switch (logn) {  // the single-mode stepper's shapes: E = 2^(logn-5) up to 2^8, then 16
        case 6: return launch_gain_t<6, 1>(desc, out, stream);
        case 7: return launch_gain_t<7, 2>(desc, out, stream);
        case 8: return launch_gain_t<8, 3>(desc, out, stream);
        case 9: return launch_gain_t<9, 4>(desc, out, stream);
        case 10: return launch_gain_t<10, 4>(desc, out, stream);
        case 11: return launch_gain_t<11, 4>(desc, out, stream);
        case 12: return launch_gain_t<12, 4>(desc, out, stream);
        case 13: return launch_gain_t<13, 4>(desc, out, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace fl
