// Self-consistent lattice on the device: the predictor, the k-average and the local
// second-order self-energy of the lattice drivers (examples/programs/hubbard_chain_2b.cpp:
// 245-324, examples/programs/gw.cpp:386-420), so that a whole lattice time step
//   extrapolate G_k -> { G_loc = <G_k>_k -> Sigma = Sigma_2B[G_loc, U] -> dyson_timestep } x ncorr
// runs without the host touching a time slice.
//   k_extrapolate  cntr::extrapolate_timestep(n, G, k) of every problem (cntr_utilities_impl.hpp:22-130)
//   k_gloc         G_loc(t) = (1/P) sum_p G_p(t), one time step, deterministic summation order
//   k_sigma_2b     Sigma(t) = Sigma_2B[G_loc, U](t) (hubbard_chain_selfen_impl.cpp:63-75) for a
//                  diagonal interaction U(t)
#pragma once
#include "kernels_dyson.cuh"

__device__ __forceinline__ double poly_interp(int k, int a, int l) {
    return c_tab.poly_interp[k][a * NESSI_K1MAX + l];
}

// ---------------------------------------------------------------------------------------
// k_extrapolate: slice n+1 of every problem with nt >= n+1 from slices n-k..n, with the
// weights p1(l) = sum_a (-1)^a poly_interpolation(a, l) (extrapolate_timestep_dispatch,
// cntr_utilities_impl.hpp:60-130).  grid.y = problem; thread per (component, element).
// Rows t' <= k of ret and les need the hermitian continuation of the stored triangles.
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_extrapolate(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    const ProbDev p = probs[blockIdx.y];
    const int n1 = n + 1;
    if (n1 > p.nt) return;
    const int k = g.k, s2 = S * S, M = g.ntau + 1;
    double p1[NESSI_K1MAX];
    for (int m = 0; m <= k; m++) {
        double v = 0.0;
        for (int l = 0; l <= k; l++) v += (l % 2 ? -1.0 : 1.0) * poly_interp(k, l, m);
        p1[m] = v;
    }
    const long ntv = (long)M * s2, nrow = (long)(n1 + 1) * s2;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ntv + 2 * nrow; e += (long)gridDim.x * blockDim.x) {
        double2 v = cmk(0, 0);
        if (e < ntv) {
            // element planes: e = ab * M + tau, row t at t * s2 * M
            for (int l = 0; l <= k; l++) v = cfma(cmk(p1[l], 0), p.gtv[(long)(n - l) * s2 * M + e], v);
            p.gtv[(long)n1 * s2 * M + e] = v;
        } else if (e < ntv + nrow) {
            const long q = e - ntv;
            const int jj = (int)(q / s2), ab = (int)(q % s2), a = ab / S, b = ab % S;
            if (jj <= k) {
                // ret(n1, j), j <= k: G^R(n-l, j) or -G^R(j, n-l)^dagger
                for (int l = 0; l <= k; l++) {
                    const int t = n - l;
                    double2 x = t <= jj ? cneg(cconj(p.gret[(tri(jj) + t) * s2 + b * S + a])) : p.gret[(tri(t) + jj) * s2 + ab];
                    v = cfma(cmk(p1[l], 0), x, v);
                }
            } else {
                // ret(n1, n1 - jr), jr = 0..n-k: along the diagonal direction
                const int jr = n1 - jj;
                for (int l = 0; l <= k; l++) {
                    const int t = n - l;
                    v = cfma(cmk(p1[l], 0), p.gret[(tri(t) + t - jr) * s2 + ab], v);
                }
            }
            p.gret[(tri(n1) + jj) * s2 + ab] = v;
        } else {
            const long q = e - ntv - nrow;
            const int j = (int)(q / s2), ab = (int)(q % s2), a = ab / S, b = ab % S;
            if (j <= k) {
                for (int l = 0; l <= k; l++) {
                    const int t = n - l;
                    double2 x = t < j ? cneg(cconj(p.gles[(tri(j) + t) * s2 + b * S + a])) : p.gles[(tri(t) + j) * s2 + ab];
                    v = cfma(cmk(p1[l], 0), x, v);
                }
            } else {
                for (int l = 0; l <= k; l++) v = cfma(cmk(p1[l], 0), p.gles[(tri(n - l) + j - l - 1) * s2 + ab], v);
            }
            p.gles[(tri(n1) + j) * s2 + ab] = v;
        }
    }
}

// ---------------------------------------------------------------------------------------
// k_gloc + k_gloc_final: G_loc(tstp) = (1/P) sum_p G_p(tstp) over the P problems of a group, as
// partial sums over chunks of 64 problems (block (32, 8): threadIdx.x = element of the slice,
// threadIdx.y = problem lane) added in a fixed order, so the result does not depend on scheduling.
// Slice elements: [ret(t,0..t) | tv planes (e*M + tau) | les(0..t,t)], or mat for tstp = -1.
// G_loc is stored in libcntr's layout (tv as ((t M + tau) s^2 + e)).
// ---------------------------------------------------------------------------------------
struct LocDev {
    double2 *ret, *les, *tv, *mat;  // G_loc, libcntr layout, ntmax / ntau / s of the group
};

#define GLOC_CHUNK 64  // problems per partial sum

// pass 1: part[c][e] = sum of element e over problems c*64 .. c*64+63 (lanes y = 0..7 take every
// 8th problem of the chunk, then the 8 lane sums are added in lane order)
template <int S>
__global__ void __launch_bounds__(256) k_gloc(GroupDev g, const ProbDev *__restrict__ probs, int nprob, int tstp,
                                              double2 *part, long ldpart) {
    __shared__ double2 red[8][32];
    const int s2 = S * S, M = g.ntau + 1;
    const long nret = tstp >= 0 ? (long)(tstp + 1) * s2 : 0, ntv = (long)M * s2;
    const long total = tstp >= 0 ? 2 * nret + ntv : ntv;
    const long e = blockIdx.x * 32L + threadIdx.x;
    const int q0 = blockIdx.y * GLOC_CHUNK, q1 = min(nprob, q0 + GLOC_CHUNK);
    double2 acc = cmk(0, 0);
    if (e < total) {
        for (int q = q0 + threadIdx.y; q < q1; q += 8) {
            const ProbDev &p = probs[q];
            double2 v;
            if (tstp < 0) v = p.gmat[e];
            else if (e < nret) v = p.gret[tri(tstp) * s2 + e];
            else if (e < nret + ntv) v = p.gtv[(long)tstp * s2 * M + (e - nret)];
            else v = p.gles[tri(tstp) * s2 + (e - nret - ntv)];
            acc = cadd(acc, v);
        }
    }
    red[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && e < total) {
        double2 v = red[0][threadIdx.x];
        for (int y = 1; y < 8; y++) v = cadd(v, red[y][threadIdx.x]);
        part[blockIdx.y * ldpart + e] = v;
    }
}

// pass 2: G_loc element e = (1/P) sum_c part[c][e], chunks in order, stored in libcntr layout
template <int S>
__global__ void k_gloc_final(GroupDev g, int nprob, int tstp, const double2 *__restrict__ part, long ldpart,
                             int nchunk, LocDev loc) {
    const int s2 = S * S, M = g.ntau + 1;
    const long nret = tstp >= 0 ? (long)(tstp + 1) * s2 : 0, ntv = (long)M * s2;
    const long total = tstp >= 0 ? 2 * nret + ntv : ntv;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        double2 v = part[e];
        for (int c = 1; c < nchunk; c++) v = cadd(v, part[c * ldpart + e]);
        v = cscale(v, 1.0 / nprob);
        if (tstp < 0) loc.mat[e] = v;
        else if (e < nret) loc.ret[tri(tstp) * s2 + e] = v;
        else if (e < nret + ntv) {
            const long q = e - nret;
            const int ab = (int)(q / M), tau = (int)(q % M);
            loc.tv[((long)tstp * M + tau) * s2 + ab] = v;
        } else loc.les[tri(tstp) * s2 + (e - nret - ntv)] = v;
    }
}

// ---------------------------------------------------------------------------------------
// k_sigma_2b: Sigma(tstp) of the group from G_loc(tstp) (libcntr layout) and a diagonal U(t)
// (udiag[(t+1) s + i], t = -1..ntmax):
//   Pol_ij = -Bubble1(G_ij, G_ij) U_i(t) U_j(t')    (Polarization + left/right_multiply)
//   Sigma_ij = Bubble2(G_ij, Pol_ij)
// following get_bubble_1_timestep / get_bubble_2_timestep (cntr_bubble_impl.hpp:33-150) with
// A = Acc = G and B = Bcc = G (Bubble1) or Pol (Bubble2).  Thread per (component, m, ij).
// ---------------------------------------------------------------------------------------
struct SigOut {
    double2 *ret, *les, *tv, *mat;  // the group's Sigma (libcntr layout)
};

// Pol_ij(tstp, m) ret and les(m, tstp) parts, before the U factors
template <int S>
__device__ __forceinline__ void pol_ret_les(const double2 *gr, const double2 *gl, int i, int j, double2 &pret,
                                            double2 &ples) {
    const int a12 = i * S + j, a21 = j * S + i;
    const double2 ii = cmk(0.0, 1.0);
    const double2 bles21_tt1 = cneg(cconj(gl[a12]));
    const double2 bgtr21_tt1 = cadd(gr[a21], bles21_tt1);
    const double2 bles21_t1t = gl[a21];
    const double2 bgtr21_t1t = cadd(cneg(cconj(gr[a12])), bles21_t1t);
    const double2 ales12_tt1 = cneg(cconj(gl[a21]));
    const double2 agtr12_tt1 = cadd(gr[a12], ales12_tt1);
    const double2 cgtr = cmul(ii, cmul(agtr12_tt1, bles21_t1t));
    const double2 cles = cmul(ii, cmul(ales12_tt1, bgtr21_t1t));
    pret = cneg(csub(cgtr, cles));
    ples = cneg(cmul(ii, cmul(gl[a12], bgtr21_tt1)));
}

template <int S>
__global__ void k_sigma_2b(GroupDev g, LocDev loc, const double2 *__restrict__ udiag, int tstp, SigOut out) {
    const int s2 = S * S, ntau = g.ntau, M = ntau + 1;
    const double2 ii = cmk(0.0, 1.0);
    const double2 *U0 = udiag;  // U(-1)
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
    if (tstp < 0) {
        const double sg = -1.0 * g.sig;
        for (long e = tid; e < (long)M * s2; e += nth) {
            const int m = (int)(e / s2), ab = (int)(e % s2), i = ab / S, j = ab % S;
            double2 c = cscale(cmul(loc.mat[(long)m * s2 + ab], loc.mat[(long)(ntau - m) * s2 + j * S + i]), sg);
            double2 pol = cmul(cmul(U0[i], cneg(c)), U0[j]);
            out.mat[(long)m * s2 + ab] = cneg(cmul(loc.mat[(long)m * s2 + ab], pol));
        }
        return;
    }
    const int n = tstp;
    const double2 *Un = udiag + (long)(n + 1) * S;
    const long nrow = (long)(n + 1) * s2;
    for (long e = tid; e < nrow + (long)M * s2; e += nth) {
        if (e < nrow) {
            const int m = (int)(e / s2), ab = (int)(e % s2), i = ab / S, j = ab % S;
            const double2 *gr = loc.ret + (tri(n) + m) * s2;
            const double2 *gl = loc.les + (tri(n) + m) * s2;
            const double2 *Um = udiag + (long)(m + 1) * S;
            double2 pr_ij, pl_ij, pr_ji, pl_ji;
            pol_ret_les<S>(gr, gl, i, j, pr_ij, pl_ij);
            pol_ret_les<S>(gr, gl, j, i, pr_ji, pl_ji);
            // U factors: ret(n,m): U_i(n) . U_j(m); les(m,n): U_i(m) . U_j(n)
            pr_ij = cmul(cmul(Un[i], pr_ij), Um[j]);
            pl_ij = cmul(cmul(Um[i], pl_ij), Un[j]);
            pl_ji = cmul(cmul(Um[j], pl_ji), Un[i]);
            (void)pr_ji;
            const int a12 = ab, a21 = j * S + i;
            const double2 bgtr12 = csub(pr_ij, cconj(pl_ji));
            const double2 agtr12 = csub(gr[a12], cconj(gl[a21]));
            const double2 cgtr = cmul(ii, cmul(agtr12, bgtr12));
            const double2 cles = cmul(ii, cmul(cconj(gl[a21]), cconj(pl_ji)));
            out.ret[(tri(n) + m) * s2 + ab] = csub(cgtr, cles);
            out.les[(tri(n) + m) * s2 + ab] = cmul(ii, cmul(gl[a12], pl_ij));
        } else {
            const long q = e - nrow;
            const int m = (int)(q / s2), ab = (int)(q % s2), i = ab / S, j = ab % S;
            const double2 gtv = loc.tv[((long)n * M + m) * s2 + ab];
            const double2 bvt = cscale(cconj(loc.tv[((long)n * M + ntau - m) * s2 + ab]), -1.0 * g.sig);
            double2 ptv = cneg(cmul(ii, cmul(gtv, bvt)));
            ptv = cmul(cmul(Un[i], ptv), U0[j]);
            out.tv[((long)n * M + m) * s2 + ab] = cmul(ii, cmul(gtv, ptv));
        }
    }
}

// ---------------------------------------------------------------------------------------
// k_distance_norm2: cntr::distance_norm2(tstp, g1, g2) (cntr_utilities_impl.hpp:607-650) on
// device herm_matrix data in libcntr's layout: the sum over the elements of time step tstp (ret
// row, tv row, les column; mat for tstp = -1) of the Frobenius norm of g1 - g2.  One block;
// every thread sums a fixed strided subset and the partial sums are added in a fixed tree, so
// the result does not depend on scheduling.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_distance_norm2(int tstp, ConvHM g1, ConvHM g2, int ntau, int s2,
                                                        double *out) {
    __shared__ double part[256];
    const int M = ntau + 1;
    const long n1 = tstp + 1;
    const long nel = tstp < 0 ? M : 2 * n1 + M;
    double acc = 0.0;
    for (long e = threadIdx.x; e < nel; e += 256) {
        const double2 *a, *b;
        if (tstp < 0) {
            a = g1.mat + e * s2; b = g2.mat + e * s2;
        } else if (e < n1) {        // ret(tstp, e)
            a = g1.ret + (tri(tstp) + e) * s2; b = g2.ret + (tri(tstp) + e) * s2;
        } else if (e < n1 + M) {    // tv(tstp, tau)
            const long tau = e - n1;
            a = g1.tv + ((long)tstp * M + tau) * s2; b = g2.tv + ((long)tstp * M + tau) * s2;
        } else {                    // les(i, tstp)
            const long i = e - n1 - M;
            a = g1.les + (tri(tstp) + i) * s2; b = g2.les + (tri(tstp) + i) * s2;
        }
        double r = 0.0;
        for (int i = 0; i < s2; i++) {
            const double dx = a[i].x - b[i].x, dy = a[i].y - b[i].y;
            r += dx * dx + dy * dy;
        }
        acc += sqrt(r);
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

// ---------------------------------------------------------------------------------------
// GW self-energy diagrams of the momentum-resolved example (examples/programs/gw_selfene_impl.cpp:
// 114-153) on device herm_matrix data in libcntr's layout, for all momenta in one launch:
//   polarisation  P_q(tstp) = -sum_k w_k Bubble1(G_{k-q}, G_k)          (get_Polarization_Bubble)
//   self-energy   Sigma_k(tstp) = sum_q w_q Bubble2(G_{k-q}, W_q)        (sigma_GW)
// element by element (C_{i1 i2} from A_{i1 i2}, B_{i1 i2}), with the bubbles of
// cntr_bubble_impl.hpp:17-130 (Bubble1: i A(t,t') B(t',t); Bubble2: i A(t,t') B(t,t'); the
// continuations to t' > t from the hermitian partners, here the functions themselves) and the
// momentum index of k - q on the grid k_i = (i - nk/2) 2 pi / nk (gw_latt_impl.cpp:46-51).
// Thread per (time index m of the slice, element); grid.y = the output momentum.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int gw_k_minus_q(int nk, int k, int q) {
    const int g = nk / 2;
    int i = (k - g) - (q - g) + g;
    i %= nk;
    return i < 0 ? i + nk : i;
}

// C_{c}(t, m), C_{c}(m, t) [ret / les] or C_{c}(t, tau) [tv] or C_{c}(tau) [mat] of Bubble1 with
// A = Acc = a, B = Bcc = b, at element c = (i1, i2) (e12) and its transpose e21
__device__ __forceinline__ void gw_bubble1(int tstp, int m, int part, const ConvHM &A, const ConvHM &B, int ntau, int s2,
                                           int e12, int e21, double sigb, double2 *c_ret, double2 *c_les) {
    const double2 I = cmk(0.0, 1.0);
    const int M = ntau + 1;
    if (tstp < 0) {
        *c_ret = cscale(cmul(A.mat[(long)m * s2 + e12], B.mat[(long)(ntau - m) * s2 + e21]), -sigb);
        return;
    }
    if (part == 0) {
        const long rt = (tri(tstp) + m) * s2, lm = (tri(tstp) + m) * s2;  // ret(t, m) and les(m, t)
        const double2 bles21_tt1 = cneg(cconj(B.les[lm + e12]));
        const double2 bgtr21_tt1 = cadd(B.ret[rt + e21], bles21_tt1);
        const double2 bles21_t1t = B.les[lm + e21];
        const double2 bgtr21_t1t = cadd(cneg(cconj(B.ret[rt + e12])), bles21_t1t);
        const double2 ales12_tt1 = cneg(cconj(A.les[lm + e21]));
        const double2 agtr12_tt1 = cadd(A.ret[rt + e12], ales12_tt1);
        *c_ret = csub(cmul(I, cmul(agtr12_tt1, bles21_t1t)), cmul(I, cmul(ales12_tt1, bgtr21_t1t)));
        *c_les = cmul(I, cmul(A.les[lm + e12], bgtr21_tt1));
    } else {
        const double2 bvt21 = cscale(cconj(B.tv[((long)tstp * M + ntau - m) * s2 + e12]), -sigb);
        *c_ret = cmul(I, cmul(A.tv[((long)tstp * M + m) * s2 + e12], bvt21));
    }
}

__device__ __forceinline__ void gw_bubble2(int tstp, int m, int part, const ConvHM &A, const ConvHM &B, int ntau, int s2,
                                           int e12, int e21, double2 *c_ret, double2 *c_les) {
    const double2 I = cmk(0.0, 1.0);
    const int M = ntau + 1;
    if (tstp < 0) {
        *c_ret = cneg(cmul(A.mat[(long)m * s2 + e12], B.mat[(long)m * s2 + e12]));
        return;
    }
    if (part == 0) {
        const long rt = (tri(tstp) + m) * s2, lm = (tri(tstp) + m) * s2;
        const double2 bgtr12 = csub(B.ret[rt + e12], cconj(B.les[lm + e21]));
        const double2 agtr12 = csub(A.ret[rt + e12], cconj(A.les[lm + e21]));
        const double2 cles = cmul(I, cmul(cconj(A.les[lm + e21]), cconj(B.les[lm + e21])));
        *c_ret = csub(cmul(I, cmul(agtr12, bgtr12)), cles);
        *c_les = cmul(I, cmul(A.les[lm + e12], B.les[lm + e12]));
    } else {
        *c_ret = cmul(I, cmul(A.tv[((long)tstp * M + m) * s2 + e12], B.tv[((long)tstp * M + m) * s2 + e12]));
    }
}

// which = 1: out[q] = P_q from G (B = G_k, A = G_{k-q}), sign -w_k;  which = 2: out[k] = Sigma_k
// from G and W (A = G_{k-q}, B = W_q), sign +w_q.  Items: m = 0..tstp for ret/les (part 0) then
// m = 0..ntau for tv (part 1); tstp = -1: m = 0..ntau of mat.
__global__ void __launch_bounds__(128) k_gw_bubbles(int which, int tstp, int nk, const ConvHM *__restrict__ G,
                                                    const ConvHM *__restrict__ W, const ConvHM *__restrict__ out,
                                                    const double *__restrict__ w, int ntau, int s, double sigb) {
    const int s2 = s * s, M = ntau + 1;
    const int o = blockIdx.y;  // output momentum
    const long nitem = tstp < 0 ? (long)M * s2 : (long)(tstp + 1 + M) * s2;
    const ConvHM C = out[o];
    for (long it = blockIdx.x * (long)blockDim.x + threadIdx.x; it < nitem; it += (long)gridDim.x * blockDim.x) {
        const int e = (int)(it % s2);
        const long mi = it / s2;
        const int part = tstp < 0 ? 0 : (mi <= tstp ? 0 : 1);
        const int m = tstp < 0 ? (int)mi : (part == 0 ? (int)mi : (int)(mi - tstp - 1));
        const int i1 = e / s, i2 = e % s, e12 = e, e21 = i2 * s + i1;
        double2 r = cmk(0, 0), l = cmk(0, 0);
        for (int x = 0; x < nk; x++) {  // x = k (polarisation) or q (self-energy)
            double2 cr = cmk(0, 0), cl = cmk(0, 0);
            if (which == 1) gw_bubble1(tstp, m, part, G[gw_k_minus_q(nk, x, o)], G[x], ntau, s2, e12, e21, sigb, &cr, &cl);
            else gw_bubble2(tstp, m, part, G[gw_k_minus_q(nk, o, x)], W[x], ntau, s2, e12, e21, &cr, &cl);
            const double f = which == 1 ? -w[x] : w[x];
            r = cfma(cmk(f, 0.0), cr, r);
            l = cfma(cmk(f, 0.0), cl, l);
        }
        if (tstp < 0) {
            C.mat[(long)m * s2 + e] = r;
        } else if (part == 0) {
            C.ret[(tri(tstp) + m) * s2 + e] = r;
            C.les[(tri(tstp) + m) * s2 + e] = l;
        } else {
            C.tv[((long)tstp * M + m) * s2 + e] = r;
        }
    }
}
