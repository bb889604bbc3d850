// dsmc_adjoint.cuh -- kernels of the smoothed model and its adjoint (see dsmc_adjoint.h).
//
// State of the smoothed model: one atom per id (0..n-1), x and v as R4 (fourth lane unused), the
// spinor psi as R4 (Re u, Im u, Re d, Im d), the survival weight w.  The adjoint state holds
// ADJ_SEEDS copies (the two loss terms), seed q of atom i at index q n + i.  A step is two launches: the recorded collisions of the step, applied by one
// thread in recorded order (collisions of different cells touch different atoms; within a cell
// the recording order is the collision order), then the per-atom move + weight update.  The
// backward pass walks segments of K steps from the end: it restores the segment's checkpoint,
// recomputes the segment storing each step's start state, then runs the adjoint steps backwards.
#ifndef DSMC_ADJOINT_CUH
#define DSMC_ADJOINT_CUH

#include "dsmc_adjoint.h"
#include "dsmc_kernels.cuh"

namespace dsmc {

template <class S> struct SmoothArgs {
    typedef typename V4T<S>::type S4;
    S4* x;
    S4* v;
    S4* psi;
    S* w;
    S* e;              // knife energy after the last step
    const int2* ij;    // recorded pairs (atom ids)
    const double* nv;  // recorded directions, 3 per pair
    const int* off;    // steps + 1 offsets into the record
    S4* vpre;          // pre-collision velocities of the recorded pairs (2 per pair)
    S4* seg_x;         // stored start states of the current segment [K][n]
    S4* seg_v;
    S4* seg_psi;
    S* seg_w;
    S4* xb;            // adjoints, ADJ_SEEDS x n each
    S4* vb;
    S4* pb;
    S* wb;
    double* theta_b;   // ADJ_SEEDS x ADJ_NPARAM accumulators
    TilePartial* partials;
    SmoothConsts<S> C;
    int n;
};

// applies the recorded collisions of step t (one thread, recorded order)
template <class S>
__global__ void sm_collide(SmoothArgs<S> A, int t, int store_pre) {
    typedef typename V4T<S>::type S4;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int k = A.off[t]; k < A.off[t + 1]; ++k) {
        const int i = A.ij[k].x, j = A.ij[k].y;
        if (i < 0 || i >= A.n || j < 0 || j >= A.n) continue;
        S4 a = A.v[i], b = A.v[j];
        if (store_pre) {
            A.vpre[2 * k] = a;
            A.vpre[2 * k + 1] = b;
        }
        S vi[3] = {a.x, a.y, a.z}, vj[3] = {b.x, b.y, b.z};
        const S nn[3] = {(S)A.nv[3 * k], (S)A.nv[3 * k + 1], (S)A.nv[3 * k + 2]};
        collide_fixed(vi, vj, nn);
        a.x = vi[0]; a.y = vi[1]; a.z = vi[2];
        b.x = vj[0]; b.y = vj[1]; b.z = vj[2];
        A.v[i] = a;
        A.v[j] = b;
    }
}

// per-atom move + weight of step t; stores the start state at slot `seg` when seg >= 0
template <class S>
__global__ void __launch_bounds__(256) sm_move(SmoothArgs<S> A, S cut, int seg, int last) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= A.n) return;
    S4 xv = A.x[i], vv = A.v[i], pv = A.psi[i];
    S w = A.w[i];
    if (seg >= 0) {
        const size_t o = (size_t)seg * A.n + i;
        A.seg_x[o] = xv;
        A.seg_v[o] = vv;
        A.seg_psi[o] = pv;
        A.seg_w[o] = w;
    }
    S x[3] = {xv.x, xv.y, xv.z}, v[3] = {vv.x, vv.y, vv.z}, p[4] = {pv.x, pv.y, pv.z, pv.w};
    const S e = smooth_step(A.C, cut, x, v, p, w);
    xv.x = x[0]; xv.y = x[1]; xv.z = x[2];
    vv.x = v[0]; vv.y = v[1]; vv.z = v[2];
    pv.x = p[0]; pv.y = p[1]; pv.z = p[2]; pv.w = p[3];
    A.x[i] = xv;
    A.v[i] = vv;
    A.psi[i] = pv;
    A.w[i] = w;
    if (last) A.e[i] = e;
}

// exact sums of w and w e per block (sum_v2 <- w, sum_B <- w e)
template <class S>
__global__ void __launch_bounds__(256) sm_sums(SmoothArgs<S> A) {
    __shared__ TilePartial red[8];
    TilePartial acc;
    zero_partial(acc);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < A.n; i += gridDim.x * 256) {
        acc.sum_v2 += fx_from((double)A.w[i]);
        acc.sum_B += fx_from((double)A.w[i] * (double)A.e[i]);
    }
    block_reduce_partial<256>(acc, red);
    if (threadIdx.x == 0) A.partials[blockIdx.x] = acc;
}

__global__ void sm_sums_final(const TilePartial* p, int nb, double* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    i128 W = 0, S = 0;
    for (int b = 0; b < nb; ++b) {
        W += p[b].sum_v2;
        S += p[b].sum_B;
    }
    out[0] = fx_to_double(W);
    out[1] = fx_to_double(S);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block sum of three doubles; the totals are valid in thread 0 (every thread must call this)
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c) {
    __shared__ double s[3][32];
    a = warp_sum_d(a);
    b = warp_sum_d(b);
    c = warp_sum_d(c);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s[0][warp] = a; s[1][warp] = b; s[2][warp] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = 0; b = 0; c = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += s[0][k]; b += s[1][k]; c += s[2][k]; }
    }
    __syncthreads();
}

// adjoint seeds at the final state (sums = (W, S)): seed 0 of L_E = (m/2) S/W/(kT0), seed 1 of
// L_N = W/N0
template <class S>
__global__ void __launch_bounds__(256) adj_seed(SmoothArgs<S> A, const double* sums, double half_m_over_kT) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    double tb0 = 0, tb1 = 0;
    if (i < A.n) {
        const double W = sums[0], Sm = sums[1];
        const double e = (double)A.e[i], w = (double)A.w[i];
        const double dEdw = half_m_over_kT * (e / W - Sm / (W * W));
        const double dEde = half_m_over_kT * w / W;
        const S4 xv = A.x[i], vv = A.v[i];
        QuadField<S> f;
        quad_field(A.C.Bp, A.C.B0, xv.x, xv.y, xv.z, true, f);
        S4 xb, vb, z;
        xb.x = (S)(dEde * (double)A.C.kappa * (double)f.g[0]);
        xb.y = (S)(dEde * (double)A.C.kappa * (double)f.g[1]);
        xb.z = (S)(dEde * (double)A.C.kappa * (double)f.g[2]);
        xb.w = (S)0;
        vb.x = (S)(dEde * 2.0 * (double)vv.x);
        vb.y = (S)(dEde * 2.0 * (double)vv.y);
        vb.z = (S)(dEde * 2.0 * (double)vv.z);
        vb.w = (S)0;
        z.x = (S)0; z.y = (S)0; z.z = (S)0; z.w = (S)0;
        A.xb[i] = xb;
        A.vb[i] = vb;
        A.pb[i] = z;
        A.wb[i] = (S)dEdw;
        A.xb[A.n + i] = z;
        A.vb[A.n + i] = z;
        A.pb[A.n + i] = z;
        A.wb[A.n + i] = (S)(1.0 / (double)A.n);
        tb0 = dEde * (double)A.C.kappa * (double)f.dabs_dBp;
        tb1 = dEde * (double)A.C.kappa * (double)f.dabs_dB0;
    }
    double unused = 0;
    block_sum3(tb0, tb1, unused);
    if (threadIdx.x == 0) {
        atomicAdd(&A.theta_b[0], tb0);
        atomicAdd(&A.theta_b[1], tb1);
    }
}

// adjoint of the per-atom part of step t (start state in segment slot seg) for both seeds; the cut
// of the step depends on the knots k0 (weight 1 - f) and k0 + 1 (weight f)
template <class S>
__global__ void __launch_bounds__(256) adj_move(SmoothArgs<S> A, S cut, int seg, int k0, double f) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    double t0[ADJ_SEEDS] = {0, 0}, t1[ADJ_SEEDS] = {0, 0}, cb[ADJ_SEEDS] = {0, 0};
    if (i < A.n) {
        const size_t o = (size_t)seg * A.n + i;
        const S4 xs = A.seg_x[o], vs = A.seg_v[o], ps = A.seg_psi[o];
        const S ws = A.seg_w[o];
        const S x0[3] = {xs.x, xs.y, xs.z}, v0[3] = {vs.x, vs.y, vs.z}, p0[4] = {ps.x, ps.y, ps.z, ps.w};
        S xb[ADJ_SEEDS][3], vb[ADJ_SEEDS][3], pb[ADJ_SEEDS][4], wb[ADJ_SEEDS], tb[ADJ_SEEDS][2], cut_b[ADJ_SEEDS];
#pragma unroll
        for (int q = 0; q < ADJ_SEEDS; ++q) {
            const S4 a = A.xb[q * A.n + i], b = A.vb[q * A.n + i], c = A.pb[q * A.n + i];
            xb[q][0] = a.x; xb[q][1] = a.y; xb[q][2] = a.z;
            vb[q][0] = b.x; vb[q][1] = b.y; vb[q][2] = b.z;
            pb[q][0] = c.x; pb[q][1] = c.y; pb[q][2] = c.z; pb[q][3] = c.w;
            wb[q] = A.wb[q * A.n + i];
            tb[q][0] = S(0); tb[q][1] = S(0);
            cut_b[q] = S(0);
        }
        smooth_step_adjoint(A.C, cut, x0, v0, p0, ws, xb, vb, pb, wb, tb, cut_b);
#pragma unroll
        for (int q = 0; q < ADJ_SEEDS; ++q) {
            S4 a, b, c;
            a.x = xb[q][0]; a.y = xb[q][1]; a.z = xb[q][2]; a.w = S(0);
            b.x = vb[q][0]; b.y = vb[q][1]; b.z = vb[q][2]; b.w = S(0);
            c.x = pb[q][0]; c.y = pb[q][1]; c.z = pb[q][2]; c.w = pb[q][3];
            A.xb[q * A.n + i] = a;
            A.vb[q * A.n + i] = b;
            A.pb[q * A.n + i] = c;
            A.wb[q * A.n + i] = wb[q];
            t0[q] = (double)tb[q][0];
            t1[q] = (double)tb[q][1];
            cb[q] = (double)cut_b[q] * A.C.cut_scale;
        }
    }
#pragma unroll
    for (int q = 0; q < ADJ_SEEDS; ++q) {
        block_sum3(t0[q], t1[q], cb[q]);
        if (threadIdx.x == 0) {
            double* th = A.theta_b + q * ADJ_NPARAM;
            atomicAdd(&th[0], t0[q]);
            atomicAdd(&th[1], t1[q]);
            atomicAdd(&th[2 + k0], cb[q] * (1.0 - f));
            if (f != 0.0 && 2 + k0 + 1 < ADJ_NPARAM) atomicAdd(&th[2 + k0 + 1], cb[q] * f);
        }
    }
}

// adjoint of the recorded collisions of step t, in reverse order
template <class S>
__global__ void sm_collide_adjoint(SmoothArgs<S> A, int t) {
    typedef typename V4T<S>::type S4;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int k = A.off[t + 1] - 1; k >= A.off[t]; --k) {
        const int i = A.ij[k].x, j = A.ij[k].y;
        if (i < 0 || i >= A.n || j < 0 || j >= A.n) continue;
        const S4 a = A.vpre[2 * k], b = A.vpre[2 * k + 1];
        const S vi[3] = {a.x, a.y, a.z}, vj[3] = {b.x, b.y, b.z};
        const S nn[3] = {(S)A.nv[3 * k], (S)A.nv[3 * k + 1], (S)A.nv[3 * k + 2]};
        for (int q = 0; q < ADJ_SEEDS; ++q) {
            S4 bi = A.vb[q * A.n + i], bj = A.vb[q * A.n + j];
            S vib[3] = {bi.x, bi.y, bi.z}, vjb[3] = {bj.x, bj.y, bj.z};
            collide_fixed_adjoint(vi, vj, nn, vib, vjb);
            bi.x = vib[0]; bi.y = vib[1]; bi.z = vib[2];
            bj.x = vjb[0]; bj.y = vjb[1]; bj.z = vjb[2];
            A.vb[q * A.n + i] = bi;
            A.vb[q * A.n + j] = bj;
        }
    }
}

// initial state of the recorded run by atom id, in double: out_x[3 id + a], out_v[3 id + a]
template <class R>
__global__ void __launch_bounds__(256) state_by_id(Args<R> A, int n, double* out_x, double* out_v, double* out_psi,
                                                   int* err) {
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= n) return;
    const int s = A.src_in[j];
    const auto q = A.pos_in[s];
    const auto v = A.vel_in[s];
    const auto w = A.psi_in[s];
    const int id = (int)lane_to_u32(q.w);
    if (id < 0 || id >= n) {
        atomicOr(err, EB_INCONSISTENT);
        return;
    }
    out_x[3 * id] = (double)q.x; out_x[3 * id + 1] = (double)q.y; out_x[3 * id + 2] = (double)q.z;
    out_v[3 * id] = (double)v.x; out_v[3 * id + 1] = (double)v.y; out_v[3 * id + 2] = (double)v.z;
    out_psi[4 * id] = (double)w.x; out_psi[4 * id + 1] = (double)w.y;
    out_psi[4 * id + 2] = (double)w.z; out_psi[4 * id + 3] = (double)w.w;
}

template <class S>
__global__ void __launch_bounds__(256) sm_load(SmoothArgs<S> A, const double* x0, const double* v0, const double* p0) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= A.n) return;
    S4 x, v, p;
    x.x = (S)x0[3 * i]; x.y = (S)x0[3 * i + 1]; x.z = (S)x0[3 * i + 2]; x.w = (S)0;
    v.x = (S)v0[3 * i]; v.y = (S)v0[3 * i + 1]; v.z = (S)v0[3 * i + 2]; v.w = (S)0;
    p.x = (S)p0[4 * i]; p.y = (S)p0[4 * i + 1]; p.z = (S)p0[4 * i + 2]; p.w = (S)p0[4 * i + 3];
    A.x[i] = x;
    A.v[i] = v;
    A.psi[i] = p;
    A.w[i] = (S)1;
}

}  // namespace dsmc

#endif  // DSMC_ADJOINT_CUH
