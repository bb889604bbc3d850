// dsmc_adjoint.cuh -- kernels of the smoothed model and its adjoint (see dsmc_adjoint.h).
//
// State of the smoothed model: one atom per id (0..n-1), x as R4 with the survival weight w in its
// fourth lane, v as R4 (fourth lane unused), the spinor psi as R4 (Re u, Im u, Re d, Im d).  The
// adjoint state holds ADJ_SEEDS copies (the two loss terms), seed q of atom i at index q n + i, the
// weight's adjoint in the fourth lane of the position's.  A step is the recorded
// collisions of the step, applied by one warp with every atom's collisions in recorded order
// (collisions of different cells touch different atoms; within a cell the recording order is the
// collision order), then the per-atom move + weight update; the collisions of the next step run in
// the move kernel's last block to finish, so a step is one launch.  The backward pass walks
// segments of K steps from the end: it restores the segment's checkpoint into the first slot of
// the segment store and recomputes the segment from slot to slot (each slot holds a step's start
// state), then runs the adjoint steps backwards, each with the adjoint of its collisions in the
// last block.  The parameter adjoints are summed per block of the adjoint kernels (one slot each,
// no atomics) and reduced in a fixed order at the end, so gradients repeat bit for bit.
#ifndef DSMC_ADJOINT_CUH
#define DSMC_ADJOINT_CUH

#include "dsmc_adjoint.h"
#include "dsmc_kernels.cuh"

namespace dsmc {

template <class S> struct SmoothArgs {
    typedef typename V4T<S>::type S4;
    S4* x;             // position, survival weight in .w
    S4* v;
    S4* psi;
    S* e;              // knife energy after the last step
    const int2* ij;    // recorded pairs (atom ids)
    const double* nv;  // recorded directions, 3 per pair
    const int* off;    // steps + 1 offsets into the record
    S4* vpre;          // pre-collision velocities of the recorded pairs (2 per pair)
    S4* seg_x;         // stored start states of the current segment [K][n]
    S4* seg_v;
    S4* seg_psi;
    S4* xb;            // adjoints, ADJ_SEEDS x n each
    S4* vb;
    S4* pb;
    double* theta_b;   // ADJ_SEEDS x ADJ_NPARAM results
    double* theta_part;  // per block of adj_seed / adj_move: ADJ_SEEDS x ADJ_NPARAM partial sums
    int* done;         // blocks of the running move / adjoint kernel finished (its last block resets it)
    TilePartial* partials;
    SmoothConsts<S> C;
    int n;
};

// The recorded collisions of step t, applied by one warp to the velocities v (n atoms): up to 32
// collisions at a time, one per lane; a collision waits while an earlier one of its batch that shares
// an atom is still pending, so every atom meets its collisions in recorded order (collisions without
// a shared atom commute: they touch different velocities).  REVERSE: the adjoint, which walks the
// step's collisions from the last and pulls the velocity adjoints of both seeds back through each.
template <class S, bool REVERSE>
__device__ void warp_collisions(const SmoothArgs<S>& A, typename V4T<S>::type* v, int t, int store_pre) {
    typedef typename V4T<S>::type S4;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int k0 = A.off[t], k1 = A.off[t + 1];
    for (int base = 0; base < k1 - k0; base += 32) {
        const int pos = base + lane;  // position in the order the collisions are applied
        const int k = REVERSE ? k1 - 1 - pos : k0 + pos;
        int i = -1, j = -1;
        if (pos < k1 - k0) {
            const int2 pr = A.ij[k];
            i = pr.x;
            j = pr.y;
        }
        int pending = (pos < k1 - k0 && i >= 0 && i < A.n && j >= 0 && j < A.n) ? 1 : 0;
        while (__any_sync(FULL, pending)) {
            bool blocked = false;
            for (int l = 0; l < 31; ++l) {
                const int pi = __shfl_sync(FULL, i, l), pj = __shfl_sync(FULL, j, l);
                const int pp = __shfl_sync(FULL, pending, l);
                if (l < lane && pp && (pi == i || pi == j || pj == i || pj == j)) blocked = true;
            }
            if (pending && !blocked) {
                const S nn[3] = {(S)A.nv[3 * k], (S)A.nv[3 * k + 1], (S)A.nv[3 * k + 2]};
                if (!REVERSE) {
                    S4 a = v[i], b = v[j];
                    if (store_pre) {
                        A.vpre[2 * k] = a;
                        A.vpre[2 * k + 1] = b;
                    }
                    S vi[3] = {a.x, a.y, a.z}, vj[3] = {b.x, b.y, b.z};
                    collide_fixed(vi, vj, nn);
                    a.x = vi[0]; a.y = vi[1]; a.z = vi[2];
                    b.x = vj[0]; b.y = vj[1]; b.z = vj[2];
                    v[i] = a;
                    v[j] = b;
                } else {
                    const S4 a = A.vpre[2 * k], b = A.vpre[2 * k + 1];
                    const S vi[3] = {a.x, a.y, a.z}, vj[3] = {b.x, b.y, b.z};
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
                pending = 0;
            }
            __syncwarp();  // this round's velocities are visible to the lanes that wait for them
        }
    }
}

// Run by every thread of a block at its end: the last block of the grid to get here applies the
// collisions of step t (REVERSE: their adjoint) once every block's writes are visible.
template <class S, bool REVERSE>
__device__ void collisions_in_last_block(const SmoothArgs<S>& A, typename V4T<S>::type* v, int t, int store_pre) {
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(A.done, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x < 32) {
        warp_collisions<S, REVERSE>(A, v, t, store_pre);
        if (threadIdx.x == 0) *A.done = 0;
    }
}

// the recorded collisions of step t on their own (one warp); slot < 0: the state arrays, else the
// segment slot
template <class S>
__global__ void sm_collide(SmoothArgs<S> A, int t, int store_pre, int slot) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    warp_collisions<S, false>(A, slot < 0 ? A.v : A.seg_v + (size_t)slot * A.n, t, store_pre);
}

// per-atom move + weight of a step.  slot < 0: the state arrays in place; else the start state in
// segment slot `slot`, the end state into slot + 1.  coll_t >= 0: the last block then applies the
// collisions of step coll_t to the end state (store_pre: keeping their pre-collision velocities).
template <class S>
__global__ void __launch_bounds__(256) sm_move(SmoothArgs<S> A, S cut, int slot, int last, int coll_t, int store_pre) {
    typedef typename V4T<S>::type S4;
    const size_t oi = slot < 0 ? 0 : (size_t)slot * A.n, oo = slot < 0 ? 0 : (size_t)(slot + 1) * A.n;
    S4* xi = slot < 0 ? A.x : A.seg_x + oi;
    S4* vi = slot < 0 ? A.v : A.seg_v + oi;
    S4* pi = slot < 0 ? A.psi : A.seg_psi + oi;
    S4* xo = slot < 0 ? A.x : A.seg_x + oo;
    S4* vo = slot < 0 ? A.v : A.seg_v + oo;
    S4* po = slot < 0 ? A.psi : A.seg_psi + oo;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < A.n; i += gridDim.x * 256) {
        S4 xv = xi[i], vv = vi[i], pv = pi[i];
        S w = xv.w;
        S x[3] = {xv.x, xv.y, xv.z}, v[3] = {vv.x, vv.y, vv.z}, p[4] = {pv.x, pv.y, pv.z, pv.w};
        const S e = smooth_step(A.C, cut, x, v, p, w);
        xv.x = x[0]; xv.y = x[1]; xv.z = x[2]; xv.w = w;
        vv.x = v[0]; vv.y = v[1]; vv.z = v[2];
        pv.x = p[0]; pv.y = p[1]; pv.z = p[2]; pv.w = p[3];
        xo[i] = xv;
        vo[i] = vv;
        po[i] = pv;
        if (last) A.e[i] = e;
    }
    if (coll_t >= 0) collisions_in_last_block<S, false>(A, vo, coll_t, store_pre);
}

// exact sums of w and w e per block (sum_v2 <- w, sum_B <- w e)
template <class S>
__global__ void __launch_bounds__(256) sm_sums(SmoothArgs<S> A) {
    __shared__ TilePartial red[8];
    TilePartial acc;
    zero_partial(acc);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < A.n; i += gridDim.x * 256) {
        const double w = (double)A.x[i].w;
        acc.sum_v2 += fx_from(w);
        acc.sum_B += fx_from(w * (double)A.e[i]);
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
    double tb0 = 0, tb1 = 0;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < A.n; i += gridDim.x * 256) {
        const double W = sums[0], Sm = sums[1];
        const S4 xv = A.x[i], vv = A.v[i];
        const double e = (double)A.e[i], w = (double)xv.w;
        const double dEdw = half_m_over_kT * (e / W - Sm / (W * W));
        const double dEde = half_m_over_kT * w / W;
        QuadField<S> f;
        quad_field(A.C.Bp, A.C.B0, xv.x, xv.y, xv.z, true, f);
        S4 xb, vb, z;
        xb.x = (S)(dEde * (double)A.C.kappa * (double)f.g[0]);
        xb.y = (S)(dEde * (double)A.C.kappa * (double)f.g[1]);
        xb.z = (S)(dEde * (double)A.C.kappa * (double)f.g[2]);
        xb.w = (S)dEdw;
        vb.x = (S)(dEde * 2.0 * (double)vv.x);
        vb.y = (S)(dEde * 2.0 * (double)vv.y);
        vb.z = (S)(dEde * 2.0 * (double)vv.z);
        vb.w = (S)0;
        z.x = (S)0; z.y = (S)0; z.z = (S)0; z.w = (S)0;
        A.xb[i] = xb;
        A.vb[i] = vb;
        A.pb[i] = z;
        z.w = (S)(1.0 / (double)A.n);
        A.xb[A.n + i] = z;
        z.w = (S)0;
        A.vb[A.n + i] = z;
        A.pb[A.n + i] = z;
        tb0 += dEde * (double)A.C.kappa * (double)f.dabs_dBp;
        tb1 += dEde * (double)A.C.kappa * (double)f.dabs_dB0;
    }
    double unused = 0;
    block_sum3(tb0, tb1, unused);
    if (threadIdx.x == 0) {  // the block's own slot (cleared before): seed 0, B' and B0
        double* th = A.theta_part + (size_t)blockIdx.x * ADJ_SEEDS * ADJ_NPARAM;
        th[0] += tb0;
        th[1] += tb1;
    }
}

// adjoint of the per-atom part of step t (start state in segment slot seg) for both seeds; the cut
// of the step depends on the knots k0 (weight 1 - f) and k0 + 1 (weight f).  Each block adds its
// parameter adjoints to its own slot; its last block to finish then pulls the velocity adjoints
// back through the step's collisions (in reverse order).  Atoms in a grid-stride loop over the grid
// adj_seed had (the same slots).
template <class S>
__global__ void __launch_bounds__(256) adj_move(SmoothArgs<S> A, S cut, int seg, int k0, double f, int t) {
    typedef typename V4T<S>::type S4;
    double t0[ADJ_SEEDS] = {0, 0}, t1[ADJ_SEEDS] = {0, 0}, cb[ADJ_SEEDS] = {0, 0};
    for (int i = blockIdx.x * 256 + threadIdx.x; i < A.n; i += gridDim.x * 256) {
        const size_t o = (size_t)seg * A.n + i;
        const S4 xs = A.seg_x[o], vs = A.seg_v[o], ps = A.seg_psi[o];
        const S ws = xs.w;
        const S x0[3] = {xs.x, xs.y, xs.z}, v0[3] = {vs.x, vs.y, vs.z}, p0[4] = {ps.x, ps.y, ps.z, ps.w};
        S xb[ADJ_SEEDS][3], vb[ADJ_SEEDS][3], pb[ADJ_SEEDS][4], wb[ADJ_SEEDS], tb[ADJ_SEEDS][2], cut_b[ADJ_SEEDS];
#pragma unroll
        for (int q = 0; q < ADJ_SEEDS; ++q) {
            const S4 a = A.xb[q * A.n + i], b = A.vb[q * A.n + i], c = A.pb[q * A.n + i];
            xb[q][0] = a.x; xb[q][1] = a.y; xb[q][2] = a.z;
            vb[q][0] = b.x; vb[q][1] = b.y; vb[q][2] = b.z;
            pb[q][0] = c.x; pb[q][1] = c.y; pb[q][2] = c.z; pb[q][3] = c.w;
            wb[q] = a.w;
            tb[q][0] = S(0); tb[q][1] = S(0);
            cut_b[q] = S(0);
        }
        smooth_step_adjoint(A.C, cut, x0, v0, p0, ws, xb, vb, pb, wb, tb, cut_b);
#pragma unroll
        for (int q = 0; q < ADJ_SEEDS; ++q) {
            S4 a, b, c;
            a.x = xb[q][0]; a.y = xb[q][1]; a.z = xb[q][2]; a.w = wb[q];
            b.x = vb[q][0]; b.y = vb[q][1]; b.z = vb[q][2]; b.w = S(0);
            c.x = pb[q][0]; c.y = pb[q][1]; c.z = pb[q][2]; c.w = pb[q][3];
            A.xb[q * A.n + i] = a;
            A.vb[q * A.n + i] = b;
            A.pb[q * A.n + i] = c;
            t0[q] += (double)tb[q][0];
            t1[q] += (double)tb[q][1];
            cb[q] += (double)cut_b[q] * A.C.cut_scale;
        }
    }
#pragma unroll
    for (int q = 0; q < ADJ_SEEDS; ++q) {
        block_sum3(t0[q], t1[q], cb[q]);
        if (threadIdx.x == 0) {
            double* th = A.theta_part + ((size_t)blockIdx.x * ADJ_SEEDS + q) * ADJ_NPARAM;
            th[0] += t0[q];
            th[1] += t1[q];
            th[2 + k0] += cb[q] * (1.0 - f);
            if (f != 0.0 && 2 + k0 + 1 < ADJ_NPARAM) th[2 + k0 + 1] += cb[q] * f;
        }
    }
    collisions_in_last_block<S, true>(A, A.v, t, 0);
}

// theta_b[o] = sum over the nb blocks' slots of output o (one warp per output, a fixed order)
__global__ void adj_theta_reduce(const double* part, int nb, double* theta_b) {
    const int o = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (o >= ADJ_SEEDS * ADJ_NPARAM) return;
    double acc = 0;
    for (int b = lane; b < nb; b += 32) acc += part[(size_t)b * ADJ_SEEDS * ADJ_NPARAM + o];
    acc = warp_sum_d(acc);
    if (lane == 0) theta_b[o] = acc;
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
    x.x = (S)x0[3 * i]; x.y = (S)x0[3 * i + 1]; x.z = (S)x0[3 * i + 2]; x.w = (S)1;
    v.x = (S)v0[3 * i]; v.y = (S)v0[3 * i + 1]; v.z = (S)v0[3 * i + 2]; v.w = (S)0;
    p.x = (S)p0[4 * i]; p.y = (S)p0[4 * i + 1]; p.z = (S)p0[4 * i + 2]; p.w = (S)p0[4 * i + 3];
    A.x[i] = x;
    A.v[i] = v;
    A.psi[i] = p;
}

}  // namespace dsmc

#endif  // DSMC_ADJOINT_CUH
