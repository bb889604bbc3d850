// dsmc_adjoint.cuh -- kernels of the smoothed model and its adjoint (see dsmc_adjoint.h).
//
// State of the smoothed model: one atom per id (0..n-1), x and v as R4 (fourth lane unused), the
// survival weight w.  A step is two launches: the recorded collisions of the step, applied by one
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
    S* w;
    S* e;              // knife energy after the last step
    const int2* ij;    // recorded pairs (atom ids)
    const double* nv;  // recorded directions, 3 per pair
    const int* off;    // steps + 1 offsets into the record
    S4* vpre;          // pre-collision velocities of the recorded pairs (2 per pair)
    S4* seg_x;         // stored start states of the current segment [K][n]
    S4* seg_v;
    S* seg_w;
    S4* xb;            // adjoints
    S4* vb;
    S* wb;
    double* theta_b;   // ADJ_NPARAM accumulators
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
    S4 xv = A.x[i], vv = A.v[i];
    S w = A.w[i];
    if (seg >= 0) {
        const size_t o = (size_t)seg * A.n + i;
        A.seg_x[o] = xv;
        A.seg_v[o] = vv;
        A.seg_w[o] = w;
    }
    S x[3] = {xv.x, xv.y, xv.z}, v[3] = {vv.x, vv.y, vv.z};
    const S e = smooth_step(A.C, cut, x, v, w);
    xv.x = x[0]; xv.y = x[1]; xv.z = x[2];
    vv.x = v[0]; vv.y = v[1]; vv.z = v[2];
    A.x[i] = xv;
    A.v[i] = vv;
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

// adjoint seeds of L = (m/2) S/W/(kT0) + W/N0 at the final state; sums = (W, S)
template <class S>
__global__ void __launch_bounds__(256) adj_seed(SmoothArgs<S> A, const double* sums, double half_m_over_kT) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    double tb0 = 0, tb1 = 0;
    if (i < A.n) {
        const double W = sums[0], Sm = sums[1];
        const double e = (double)A.e[i], w = (double)A.w[i];
        const double dLdw = half_m_over_kT * (e / W - Sm / (W * W)) + 1.0 / (double)A.n;
        const double dLde = half_m_over_kT * w / W;
        const S4 xv = A.x[i], vv = A.v[i];
        QuadField<S> f;
        quad_field(A.C.Bp, A.C.B0, xv.x, xv.y, xv.z, true, f);
        S4 xb, vb;
        xb.x = (S)(dLde * (double)A.C.kappa * (double)f.g[0]);
        xb.y = (S)(dLde * (double)A.C.kappa * (double)f.g[1]);
        xb.z = (S)(dLde * (double)A.C.kappa * (double)f.g[2]);
        xb.w = (S)0;
        vb.x = (S)(dLde * 2.0 * (double)vv.x);
        vb.y = (S)(dLde * 2.0 * (double)vv.y);
        vb.z = (S)(dLde * 2.0 * (double)vv.z);
        vb.w = (S)0;
        A.xb[i] = xb;
        A.vb[i] = vb;
        A.wb[i] = (S)dLdw;
        tb0 = dLde * (double)A.C.kappa * (double)f.dabs_dBp;
        tb1 = dLde * (double)A.C.kappa * (double)f.dabs_dB0;
    }
    double unused = 0;
    block_sum3(tb0, tb1, unused);
    if (threadIdx.x == 0) {
        atomicAdd(&A.theta_b[0], tb0);
        atomicAdd(&A.theta_b[1], tb1);
    }
}

// adjoint of the per-atom part of step t (start state in segment slot seg); the cut of the step
// depends on the knots k0 (weight 1 - f) and k0 + 1 (weight f)
template <class S>
__global__ void __launch_bounds__(256) adj_move(SmoothArgs<S> A, S cut, int seg, int k0, double f) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    double t0 = 0, t1 = 0, cb = 0;
    if (i < A.n) {
        const size_t o = (size_t)seg * A.n + i;
        const S4 xs = A.seg_x[o], vs = A.seg_v[o];
        const S ws = A.seg_w[o];
        const S x0[3] = {xs.x, xs.y, xs.z}, v0[3] = {vs.x, vs.y, vs.z};
        S4 xbv = A.xb[i], vbv = A.vb[i];
        S xb[3] = {xbv.x, xbv.y, xbv.z}, vb[3] = {vbv.x, vbv.y, vbv.z};
        S wb = A.wb[i];
        S tb[2] = {S(0), S(0)};
        S cut_b = S(0);
        smooth_step_adjoint(A.C, cut, x0, v0, ws, xb, vb, wb, tb, cut_b);
        xbv.x = xb[0]; xbv.y = xb[1]; xbv.z = xb[2];
        vbv.x = vb[0]; vbv.y = vb[1]; vbv.z = vb[2];
        A.xb[i] = xbv;
        A.vb[i] = vbv;
        A.wb[i] = wb;
        t0 = (double)tb[0];
        t1 = (double)tb[1];
        cb = (double)cut_b * A.C.cut_scale;
    }
    block_sum3(t0, t1, cb);
    if (threadIdx.x == 0) {
        atomicAdd(&A.theta_b[0], t0);
        atomicAdd(&A.theta_b[1], t1);
        atomicAdd(&A.theta_b[2 + k0], cb * (1.0 - f));
        if (f != 0.0 && 2 + k0 + 1 < ADJ_NPARAM) atomicAdd(&A.theta_b[2 + k0 + 1], cb * f);
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
        S4 bi = A.vb[i], bj = A.vb[j];
        S vib[3] = {bi.x, bi.y, bi.z}, vjb[3] = {bj.x, bj.y, bj.z};
        collide_fixed_adjoint(vi, vj, nn, vib, vjb);
        bi.x = vib[0]; bi.y = vib[1]; bi.z = vib[2];
        bj.x = vjb[0]; bj.y = vjb[1]; bj.z = vjb[2];
        A.vb[i] = bi;
        A.vb[j] = bj;
    }
}

// initial state of the recorded run by atom id, in double: out_x[3 id + a], out_v[3 id + a]
template <class R>
__global__ void __launch_bounds__(256) state_by_id(Args<R> A, int n, double* out_x, double* out_v, int* err) {
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= n) return;
    const int s = A.src_in[j];
    const auto q = A.pos_in[s];
    const auto v = A.vel_in[s];
    const int id = (int)lane_to_u32(q.w);
    if (id < 0 || id >= n) {
        atomicOr(err, EB_INCONSISTENT);
        return;
    }
    out_x[3 * id] = (double)q.x; out_x[3 * id + 1] = (double)q.y; out_x[3 * id + 2] = (double)q.z;
    out_v[3 * id] = (double)v.x; out_v[3 * id + 1] = (double)v.y; out_v[3 * id + 2] = (double)v.z;
}

template <class S>
__global__ void __launch_bounds__(256) sm_load(SmoothArgs<S> A, const double* x0, const double* v0) {
    typedef typename V4T<S>::type S4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= A.n) return;
    S4 x, v;
    x.x = (S)x0[3 * i]; x.y = (S)x0[3 * i + 1]; x.z = (S)x0[3 * i + 2]; x.w = (S)0;
    v.x = (S)v0[3 * i]; v.y = (S)v0[3 * i + 1]; v.z = (S)v0[3 * i + 2]; v.w = (S)0;
    A.x[i] = x;
    A.v[i] = v;
    A.w[i] = (S)1;
}

}  // namespace dsmc

#endif  // DSMC_ADJOINT_CUH
