// Depth-node form of the mixed single-slab Bethe-Heitler + Elwert scorer.
//
// The per-(segment, energy) form (pb_brem.cu, brem.py:829-1239) evaluates,
// for every segment s and photon energy k,
//   spec[d][k] += (c0 / k) sum_el w_el(s) J_el(T_s, k) Tbar_d(s, k),
// with w_el = n_el L Z_el^2 den_i(T_s), J_el the electron-energy part of the
// cross section (beta_i / p_i^2 ln((p_i + p_f)/(p_i - p_f)) / beta_f /
// (1 - exp(-2 pi alpha Z_el / beta_f))), and Tbar_d the segment-mean escape
// exp(-mu(k) f_d z') over the segment's depth extent [a_s, b_s] below the exit
// face (f_d = 1/|n_z,d|). Both factors that couple a segment to an energy are
// smooth in one segment variable each, so the double sum factorises:
//
//  * Electron energy. The segments whose T lies in a window [T_lo, T_hi]
//    just below the batch's highest T (T_hi / T_lo <= 1.1, T_lo >= 2.5 k_max)
//    see J_el(T, k) as a degree-5 polynomial in u = (T - T_c) / T_h, fitted at
//    six Chebyshev nodes per (energy, element) and checked at five other
//    points to 1e-7 (else the launch falls back to the per-pair form).
//  * Depth. exp(-lambda z') on cell c of a depth grid is the degree-7
//    polynomial through eight Chebyshev nodes of the cell, whose error is at
//    most (lambda h / 2)^8 e^(lambda h) / (2^7 8!) of the cell's smallest
//    value. The first five cells are h_min = 1/lambda_max wide (lambda_max =
//    max_k mu f_max, so lambda h <= 1: below 2e-9); deeper cells start at z
//    and are 0.2 z wide, where for any lambda the error against the surface
//    value, (0.1 lambda z)^8 e^(-0.8 lambda z) / (2^7 8!), stays below
//    6.5e-11. The segment mean of a polynomial is exact: mean_t t^j over the
//    segment's overlap with a cell, from the cancellation-free divided
//    difference D_{j+1}(t_a, t_b) = sum_i t_b^i t_a^(j-i).
//
// So one pass over the segments accumulates, per (element, face, cell), the
// moments S[p][j] = sum_s w_el u^p mean(t^j) (48 per cell), and one block per
// photon energy contracts them:
//   spec[d][k] += (c0 / k) sum_c sum_i exp(-mu f_d z_ci) W_ci,
//   W_ci = sum_j Lm[i][j] sum_el sum_p A_el,p(k) S_el,face(d),c[p][j],
// Lm the Lagrange basis of the cell nodes in monomials. The work per segment
// no longer depends on the number of energies, and the 16 detector tiles need
// no direction moments. Segments outside the window (and all of them when a
// check fails) go through a list to the per-pair kernels.
#include <cstdint>

#include "pb_brem_node.cuh"
#include "pb_common.cuh"

namespace pb {

namespace {

constexpr double kNodeMc2 = 510.99895;
constexpr int kNodeThreads = 256;
constexpr int kContractThreads = 128;
constexpr int kNodeTile = 2048;  // segments a block orders by depth cell at a time (1024: 7 % slower, 4096: 3 %)

__device__ __forceinline__ bool node_radiates(const pb_brem_args &a, int64_t s) {
    return a.elec_id[s] < a.Ne && (a.seg_layer == nullptr || a.seg_layer[s] == a.emit_layer);
}

__device__ __forceinline__ int64_t node_live(const pb_brem_args &a) {
    int64_t live = a.n_seg;
    if (a.n_seg_device && (int64_t)*a.n_seg_device < live) live = (int64_t)*a.n_seg_device;
    return live;
}

// J_el(T, k) in FP64 (the per-pair FP64 form without w_el and c0 / k; the
// born logarithm from (p_i + p_f)^2 / (p_i^2 - p_f^2), p_i^2 - p_f^2 =
// k (T + T_f + 2 m c^2) / (m c^2)^2, without cancellation).
__device__ double node_J(double T, double k, double Z) {
    const double Tf = T - k;
    if (!(Tf > 0.0) || !(k > 0.0)) return 0.0;
    const double p_i = sqrt(T * (T + 2.0 * kNodeMc2)) / kNodeMc2;
    const double b_i = p_i / (1.0 + T / kNodeMc2);
    const double p_f = sqrt(Tf * (Tf + 2.0 * kNodeMc2)) / kNodeMc2;
    const double b_f = p_f / (1.0 + Tf / kNodeMc2);
    const double dpp = k * (T + Tf + 2.0 * kNodeMc2) / (kNodeMc2 * kNodeMc2);
    const double s = p_i + p_f;
    const double bl = log(s * s / dpp);
    return b_i / (p_i * p_i) * bl / b_f / (1.0 - exp(-2.0 * kPi * kAlphaFs * Z / b_f));
}

// Cell of depth z (boundaries zb, n cells): the closed form of the grid, then
// a step either way against the stored boundaries.
__device__ __forceinline__ int node_cell(const double *zb, int n, double h_min, double z_g, double z) {
    int c;
    if (z < z_g) c = (int)(z / h_min);
    else c = kNodeUniform + (int)(log(z / z_g) * (1.0 / log(kNodeGrowth)));
    c = c < 0 ? 0 : (c > n - 1 ? n - 1 : c);
    while (c > 0 && z < zb[c]) --c;
    while (c < n - 1 && z >= zb[c + 1]) ++c;
    return c;
}

// Extent of the launch: the largest and smallest electron energy of the
// radiating segments.
__global__ void __launch_bounds__(kNodeThreads) brem_node_range_kernel(const pb_brem_args a, BremNodeHdr *h) {
    const int64_t live = node_live(a);
    unsigned long long mx = 0ULL, mnc = 0ULL;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < live;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (!node_radiates(a, s)) continue;
        const double T = a.E_keV[s];
        if (!(T > 0.0 && T < 1e300)) continue;
        const unsigned long long b = (unsigned long long)__double_as_longlong(T);
        mx = b > mx ? b : mx;
        mnc = ~b > mnc ? ~b : mnc;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, mx, o);
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, mnc, o);
        mx = x > mx ? x : mx;
        mnc = y > mnc ? y : mnc;
    }
    if ((threadIdx.x & 31) == 0 && mx != 0ULL) {
        atomicMax(&h->t_max_bits, mx);
        atomicMax(&h->t_minc_bits, mnc);
    }
}

// The window, the depth grid, its nodes and the Lagrange basis (one block).
__global__ void __launch_bounds__(kNodeThreads) brem_node_setup_kernel(const pb_brem_args a, BremNodeHdr *h) {
    __shared__ double red[2][kNodeThreads / 32];
    const int tid = threadIdx.x;
    double kmax = 0.0, mumax = 0.0;
    bool finite = true;
    for (int e = tid; e < a.n_E; e += blockDim.x) {
        kmax = fmax(kmax, a.E_grid[e] / 1e3);
        const double m = a.mu[e];
        finite = finite && m >= 0.0 && m < 1e300;
        mumax = fmax(mumax, m);
    }
    const bool all_finite = __syncthreads_and(finite);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kmax = fmax(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
        mumax = fmax(mumax, __shfl_xor_sync(0xffffffffu, mumax, o));
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = kmax;
        red[1][tid >> 5] = mumax;
    }
    __syncthreads();
    __shared__ int n_s, ok_s;
    if (tid == 0) {
        for (int w = 0; w < kNodeThreads / 32; ++w) {
            kmax = fmax(kmax, red[0][w]);
            mumax = fmax(mumax, red[1][w]);
        }
        double f_max = 0.0;
        unsigned int faces = 0u;
        for (int d = 0; d < a.n_dir; ++d) {
            const double nz = a.n_hat[3 * d + 2];
            f_max = fmax(f_max, 1.0 / fmax(fabs(nz), 1.0e-12));
            faces |= nz < 0.0 ? 1u : 2u;
        }
        bool ok = h->t_max_bits != 0ULL && all_finite;
        const double T_hi = __longlong_as_double((long long)h->t_max_bits);
        const double T_min = __longlong_as_double((long long)~h->t_minc_bits);
        const double T_lo = fmax(T_min, fmax(T_hi / kNodeWindow, kNodeTip * kmax));
        ok = ok && T_lo <= T_hi;
        const double T_slab = a.thickness;
        ok = ok && T_slab > 0.0;
        const double lam = mumax * f_max;
        const double h_min = lam > 0.0 ? fmin(1.0 / lam, T_slab) : T_slab;
        const double z_g = kNodeUniform * h_min;
        int n = 0;
        h->zb[0] = 0.0;
        while (ok && h->zb[n] < T_slab) {
            if (n == kNodeMaxCells) {
                ok = false;
                break;
            }
            ++n;
            h->zb[n] = n <= kNodeUniform ? n * h_min : z_g * pow(kNodeGrowth, (double)(n - kNodeUniform));
        }
        if (ok) h->zb[n] = T_slab;
        h->n_cells = ok ? n : 0;
        h->faces = faces;
        h->T_lo = T_lo;
        h->T_hi = T_hi;
        h->Tc = 0.5 * (T_lo + T_hi);
        h->Th = 0.5 * (T_hi - T_lo);
        h->h_min = h_min;
        h->z_g = z_g;
        n_s = ok ? n : 0;
        ok_s = ok ? 1 : 0;
    }
    __syncthreads();
    if (!ok_s) return;  // h->ok stays 0 (the workspace was zeroed)
    const int n = n_s;
    // the cells' Chebyshev nodes
    for (int q = tid; q < n * kNodePts; q += blockDim.x) {
        const int c = q / kNodePts, i = q - c * kNodePts;
        const double mid = 0.5 * (h->zb[c] + h->zb[c + 1]), hw = 0.5 * (h->zb[c + 1] - h->zb[c]);
        h->node[q] = mid + hw * cos((2 * i + 1) * kPi / (2 * kNodePts));
    }
    // Lagrange basis of the Chebyshev nodes x_i: l_i(t) = (1/n) [1 + 2 sum_m T_m(x_i) T_m(t)],
    // with T_m in monomials from T_{m+1} = 2 t T_m - T_{m-1}.
    if (tid < kNodePts * kNodePts) {
        const int i = tid / kNodePts, j = tid - i * kNodePts;
        double Tc[kNodePts][kNodePts] = {};
        Tc[0][0] = 1.0;
        Tc[1][1] = 1.0;
        for (int m = 1; m + 1 < kNodePts; ++m)
            for (int k = 0; k < kNodePts; ++k) Tc[m + 1][k] = (k > 0 ? 2.0 * Tc[m][k - 1] : 0.0) - Tc[m - 1][k];
        double v = 0.0;
        for (int m = 0; m < kNodePts; ++m)
            v += (m == 0 ? 1.0 : 2.0) / kNodePts * cos(m * (2 * i + 1) * kPi / (2 * kNodePts)) * Tc[m][j];
        h->Lm[tid] = v;
    }
    __syncthreads();
    if (tid == 0) h->ok = 1u;
}

// J_el over the window as a degree-5 polynomial in u, per (energy, element):
// Chebyshev coefficients from six nodes, then monomials; checked against J
// at u = -1, -1/2, 0, 1/2, 1 to 1e-7 (a miss turns the node form off).
__global__ void brem_node_fit_kernel(const pb_brem_args a, BremNodeHdr *h, double *A) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n_E * a.n_el || !h->ok) return;
    const int e = q / a.n_el, el = q - e * a.n_el;
    const double k = a.E_grid[e] / 1e3, Z = a.Z[el];
    const double Tc = h->Tc, Th = h->Th;
    double *out = A + (int64_t)q * kNodeTDeg;
    if (!(k > 0.0)) {
        for (int p = 0; p < kNodeTDeg; ++p) out[p] = 0.0;
        return;
    }
    double f[kNodeTDeg];
    for (int m = 0; m < kNodeTDeg; ++m) f[m] = node_J(Tc + Th * cos((2 * m + 1) * kPi / (2 * kNodeTDeg)), k, Z);
    double c[kNodeTDeg];
    for (int p = 0; p < kNodeTDeg; ++p) {
        double v = 0.0;
        for (int m = 0; m < kNodeTDeg; ++m) v += f[m] * cos(p * (2 * m + 1) * kPi / (2 * kNodeTDeg));
        c[p] = v * (p == 0 ? 1.0 : 2.0) / kNodeTDeg;
    }
    // T_0..T_5 in monomials
    const double A0 = c[0] - c[2] + c[4], A1 = c[1] - 3.0 * c[3] + 5.0 * c[5], A2 = 2.0 * c[2] - 8.0 * c[4];
    const double A3 = 4.0 * c[3] - 20.0 * c[5], A4 = 8.0 * c[4], A5 = 16.0 * c[5];
    out[0] = A0;
    out[1] = A1;
    out[2] = A2;
    out[3] = A3;
    out[4] = A4;
    out[5] = A5;
    bool good = true;
    for (int t = 0; t < 5; ++t) {
        const double u = -1.0 + 0.5 * t;
        const double ex = node_J(Tc + Th * u, k, Z);
        const double pv = ((((A5 * u + A4) * u + A3) * u + A2) * u + A1) * u + A0;
        good = good && fabs(pv - ex) <= 1e-7 * fabs(ex);
    }
    if (!good) atomicExch(&h->ok, 0u);
}

// D += A B on the FP64 tensor cores, one m8n8k4 tile: lane l holds
// A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One pass over the segments, a warp per group of 32 consecutive segments, a
// lane per segment. Each lane tests its segment against the window (the
// others are appended to the left-out list, one atomic per warp) and forms
// its weights w_el u^p and each face's depth extent. Then the lanes walk
// their segments' cells in rounds: in each round every lane with a piece left
// forms the piece's eight depth moments mean(t^j), and the lanes whose pieces
// share a cell add their outer products w_el u^p x mean(t^j) in one FP64
// tensor-core product (the 6 x 32 weights times the 32 x 8 moments, as eight
// m8n8k4 steps over the lanes); 48 lanes' worth of sums then go to the
// block's float accumulator in shared memory, one address per lane.
// Consecutive segments come from one transport step of neighbouring
// histories, so a round's pieces mostly share a cell and a warp issues a few
// tensor-core products per round. The block's sums are folded into the FP64
// moments at the end.
constexpr int kNodeWarps = kNodeThreads / 32;

// Dynamic shared memory of the moment pass: the block's float accumulator,
// then per warp the lanes' weights and piece moments.
constexpr int kNodeRow = kNodePts + 1;  // padded row of the staged weights and moments (2-way bank conflicts)
__host__ __device__ constexpr size_t node_accum_smem(int n_el) {
    return sizeof(double) * (size_t)kNodeWarps * (n_el + 1) * 32 * kNodeRow +
           sizeof(float) * (size_t)n_el * 2 * kNodeMaxCells * kNodePJ;
}

template <int NEL>
__global__ void __launch_bounds__(kNodeThreads, 2) brem_node_accum_kernel(const pb_brem_args a, BremNodeHdr *h,
                                                                           double *S, int64_t *idx, int64_t cap) {
    constexpr int kWarps = kNodeWarps;
    extern __shared__ __align__(16) unsigned char node_smem[];
    // weights w_el u^p of each lane's piece (p < 6) and its depth moments
    double (*sW)[NEL][32][kNodeRow] = reinterpret_cast<double (*)[NEL][32][kNodeRow]>(node_smem);
    double (*sM)[32][kNodeRow] =
        reinterpret_cast<double (*)[32][kNodeRow]>(node_smem + sizeof(double) * kWarps * NEL * 32 * kNodeRow);
    float *Ss = reinterpret_cast<float *>(node_smem + sizeof(double) * kWarps * (NEL + 1) * 32 * kNodeRow);
    __shared__ double zb_s[kNodeMaxCells + 1];
    __shared__ double mid_s[kNodeMaxCells], ihw_s[kNodeMaxCells];  // cell centre and 2 / width
    __shared__ unsigned short ord_s[kNodeTile];   // the tile's window segments in cell order
    __shared__ unsigned char key_s[kNodeTile];    // start cell per segment (kNodeMaxCells: not in the window)
    __shared__ int cnt_s[kNodeMaxCells + 1];
    __shared__ int n_in_s;
    __shared__ double prm[6];
    __shared__ int go_s, nc_s;
    __shared__ unsigned int faces_s;
    const int tid = threadIdx.x;
    if (tid == 0) {
        go_s = h->ok ? 1 : 0;
        nc_s = h->n_cells;
        faces_s = h->faces;
        prm[0] = h->T_lo;
        prm[1] = h->T_hi;
        prm[2] = h->Tc;
        prm[3] = h->Th > 0.0 ? 1.0 / h->Th : 0.0;
        prm[4] = h->h_min;
        prm[5] = h->z_g;
    }
    __syncthreads();
    if (!go_s) return;
    const int nc = nc_s;
    const unsigned int faces = faces_s;
    for (int c = tid; c <= nc; c += blockDim.x) zb_s[c] = h->zb[c];
    for (int c = tid; c < nc; c += blockDim.x) {
        mid_s[c] = 0.5 * (h->zb[c] + h->zb[c + 1]);
        ihw_s[c] = 2.0 / (h->zb[c + 1] - h->zb[c]);
    }
    for (int q = tid; q < NEL * 2 * kNodeMaxCells * kNodePJ; q += blockDim.x) Ss[q] = 0.0f;
    __syncthreads();
    const double T_lo = prm[0], T_hi = prm[1], Tc = prm[2], inv_Th = prm[3], h_min = prm[4], z_g = prm[5];
    const double T_slab = a.thickness;
    const double za = 2.0 * kPi * kAlphaFs;
    const int64_t live = node_live(a);
    const unsigned int lane = tid & 31;
    const int warp = tid >> 5;
    const int grow = (int)(lane >> 2), gcol = (int)(lane & 3);  // tile row / column group of this lane
    constexpr double kInvJ1[kNodePts] = {1.0, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8};
    // Tiles of kNodeTile consecutive segments, ordered by the depth cell of
    // their start on the first face in use (a counting sort in shared
    // memory), so that the 32 segments a warp takes share their cells and a
    // round of pieces needs one or two tensor-core products.
    const int f0 = (faces & 1u) ? 0 : 1;
    const int64_t n_tiles = (live + kNodeTile - 1) / kNodeTile;
    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int64_t t0 = tile * kNodeTile;
        for (int q = tid; q <= kNodeMaxCells; q += blockDim.x) cnt_s[q] = 0;
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < kNodeTile / kNodeThreads; ++k) {
            const int li = k * kNodeThreads + tid;
            const int64_t s = t0 + li;
            const bool rad = s < live && node_radiates(a, s);
            const double T = rad ? a.E_keV[s] : 0.0;
            const bool in_win = rad && T >= T_lo && T <= T_hi;
            const bool left = rad && !in_win;
            const unsigned int lm = __ballot_sync(0xffffffffu, left);
            if (lm) {
                const int ld = __ffs(lm) - 1;
                unsigned long long q0 = 0ULL;
                if ((int)lane == ld) q0 = atomicAdd(&h->n_out, (unsigned long long)__popc(lm));
                q0 = __shfl_sync(0xffffffffu, q0, ld);
                if (left) {
                    const unsigned long long q = q0 + (unsigned long long)__popc(lm & ((1u << lane) - 1u));
                    if (q < (unsigned long long)cap) idx[q] = s;
                    else atomicExch(&h->ok, 0u);  // list full: the per-pair form takes every segment
                }
            }
            int key = kNodeMaxCells;  // outside the window: after every cell
            if (in_win) {
                const double half = 0.5 * a.L[s];
                const double zm = a.r_mid[3 * s + 2], vz = a.v_hat[3 * s + 2];
                const double d0 = fmin(fmax(zm - half * vz, 0.0), T_slab);
                const double d1 = fmin(fmax(zm + half * vz, 0.0), T_slab);
                const double zs = f0 == 0 ? fmin(d0, d1) : T_slab - fmax(d0, d1);
                key = node_cell(zb_s, nc, h_min, z_g, zs);
            }
            key_s[li] = (unsigned char)key;
            atomicAdd(&cnt_s[key], 1);
        }
        __syncthreads();
        if (tid == 0) {
            int run = 0;
            for (int c = 0; c <= kNodeMaxCells; ++c) {
                const int v = cnt_s[c];
                cnt_s[c] = run;
                run += v;
            }
            n_in_s = cnt_s[kNodeMaxCells];
        }
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < kNodeTile / kNodeThreads; ++k) {
            const int li = k * kNodeThreads + tid;
            const int pos = atomicAdd(&cnt_s[key_s[li]], 1);
            ord_s[pos] = (unsigned short)li;
        }
        __syncthreads();
        const int n_in = n_in_s;
        for (int g = warp; g * 32 < n_in; g += kWarps) {
            const int pos = g * 32 + (int)lane;
            const bool in_win = pos < n_in;
            const int64_t s = in_win ? t0 + ord_s[pos] : 0;
            const double T = in_win ? a.E_keV[s] : 0.0;
            double lo = 0.0, hi = 0.0;
            if (in_win) {
                const double u = (T - Tc) * inv_Th;
                // 1 / beta_i = (T + m c^2) / sqrt(T (T + 2 m c^2))
                const double inv_bi = (T + kNodeMc2) / sqrt(T * (T + 2.0 * kNodeMc2));
                const double Lc = a.L[s];
    #pragma unroll
                for (int el = 0; el < NEL; ++el) {
                    const double Z = a.Z[el];
                    double wp = a.n_ang3[el] * 1e24 * (Lc * 1e-8) * (Z * Z) * (1.0 - exp(-za * Z * inv_bi));
    #pragma unroll
                    for (int p = 0; p < kNodePts; ++p) {
                        sW[warp][el][lane][p] = p < kNodeTDeg ? wp : 0.0;
                        wp *= u;
                    }
                }
                const double half = 0.5 * Lc;
                const double zm = a.r_mid[3 * s + 2], vz = a.v_hat[3 * s + 2];
                const double d0 = fmin(fmax(zm - half * vz, 0.0), T_slab);
                const double d1 = fmin(fmax(zm + half * vz, 0.0), T_slab);
                lo = fmin(d0, d1);
                hi = fmax(d0, d1);
            }
    #pragma unroll
            for (int f = 0; f < 2; ++f) {
                if (!((faces >> f) & 1u)) continue;
                const double za_ = f == 0 ? lo : T_slab - hi;
                const double zb_ = f == 0 ? hi : T_slab - lo;
                int c = 0, cend = -1;
                bool point = false;
                double inv_len = 0.0;
                if (in_win) {
                    c = node_cell(zb_s, nc, h_min, z_g, za_);
                    point = !(zb_ - za_ > 1e-9 * (zb_s[c + 1] - zb_s[c]));
                    cend = point ? c : node_cell(zb_s, nc, h_min, z_g, zb_);
                    inv_len = point ? 0.0 : 1.0 / (zb_ - za_);
                }
                while (__any_sync(0xffffffffu, c <= cend)) {
                    const bool have = c <= cend;
                    double M[kNodePts];
    #pragma unroll
                    for (int j = 0; j < kNodePts; ++j) M[j] = 0.0;
                    if (have) {
                        const double mid = mid_s[c], ihw = ihw_s[c];
                        if (point) {
                            const double t = fmin(fmax((za_ - mid) * ihw, -1.0), 1.0);
                            M[0] = 1.0;
    #pragma unroll
                            for (int j = 1; j < kNodePts; ++j) M[j] = M[j - 1] * t;
                        } else {
                            const double oa = fmax(za_, zb_s[c]), ob = fmin(zb_, zb_s[c + 1]);
                            if (ob > oa) {
                                const double ta = fmin(fmax((oa - mid) * ihw, -1.0), 1.0);
                                const double tb = fmin(fmax((ob - mid) * ihw, -1.0), 1.0);
                                const double frac = (ob - oa) * inv_len;
                                // D_1 = 1, D_{n+1} = t_b D_n + t_a^n; mean of t^j = frac D_{j+1} / (j + 1)
                                double D = 1.0, tan = ta;
                                M[0] = frac;
    #pragma unroll
                                for (int j = 1; j < kNodePts; ++j) {
                                    D = fma(tb, D, tan);
                                    tan *= ta;
                                    M[j] = frac * D * kInvJ1[j];
                                }
                            }
                        }
                    }
    #pragma unroll
                    for (int j = 0; j < kNodePts; ++j) sM[warp][lane][j] = M[j];
                    __syncwarp();
                    const int key = have ? c : -1;
                    unsigned int pending = __ballot_sync(0xffffffffu, have);
                    while (pending) {
                        const int ld = __ffs(pending) - 1;
                        const int K = __shfl_sync(0xffffffffu, key, ld);
                        const unsigned int grp = __ballot_sync(0xffffffffu, have && key == K);
                        pending &= ~grp;
    #pragma unroll
                        for (int el = 0; el < NEL; ++el) {
                            double d0 = 0.0, d1 = 0.0;
    #pragma unroll
                            for (int st = 0; st < 8; ++st) {
                                const int l = 4 * st + gcol;
                                const double av = ((grp >> l) & 1u) ? sW[warp][el][l][grow] : 0.0;
                                dmma_884(d0, d1, av, sM[warp][l][grow]);
                            }
                            if (grow < kNodeTDeg) {
                                float *row = Ss + ((el * 2 + f) * kNodeMaxCells + K) * kNodePJ + grow * kNodePts + 2 * gcol;
                                if (d0 != 0.0) atomicAdd(row, (float)d0);
                                if (d1 != 0.0) atomicAdd(row + 1, (float)d1);
                            }
                        }
                    }
                    __syncwarp();
                    ++c;
                }
            }
        }
        __syncthreads();  // the next tile reuses the order
    }
    __syncthreads();
    const int per = nc * kNodePJ;
    for (int q = tid; q < NEL * 2 * per; q += blockDim.x) {
        const int ef = q / per, r = q - ef * per;
        if (!((faces >> (ef & 1)) & 1u)) continue;
        const int off = ef * kNodeMaxCells * kNodePJ + r;
        const float v = Ss[off];
        if (v != 0.0f) atomicAdd(&S[off], (double)v);
    }
}

// One block per photon energy: W_ci from the moments, then every direction's
// sum over the cells' nodes.
template <int NEL>
__global__ void __launch_bounds__(kContractThreads) brem_node_contract_kernel(const pb_brem_args a,
                                                                              const BremNodeHdr *h, const double *A,
                                                                              const double *S) {
    __shared__ double W[2][kNodeMaxCells][kNodePts];
    __shared__ double nd_s[kNodeMaxCells * kNodePts];
    __shared__ double Lm_s[kNodePts * kNodePts];
    __shared__ double A_s[NEL][kNodeTDeg];
    __shared__ int go_s, nc_s;
    __shared__ unsigned int faces_s;
    const int tid = threadIdx.x;
    const int e = blockIdx.x;
    if (tid == 0) {
        go_s = (h->ok && a.E_grid[e] > 0.0) ? 1 : 0;
        nc_s = h->n_cells;
        faces_s = h->faces;
    }
    __syncthreads();
    if (!go_s) return;
    const int nc = nc_s;
    const unsigned int faces = faces_s;
    for (int q = tid; q < nc * kNodePts; q += blockDim.x) nd_s[q] = h->node[q];
    for (int q = tid; q < kNodePts * kNodePts; q += blockDim.x) Lm_s[q] = h->Lm[q];
    for (int q = tid; q < NEL * kNodeTDeg; q += blockDim.x)
        A_s[q / kNodeTDeg][q % kNodeTDeg] = A[(int64_t)e * NEL * kNodeTDeg + q];
    __syncthreads();
    for (int q = tid; q < 2 * nc; q += blockDim.x) {
        const int f = q / nc, c = q - f * nc;
        if (!((faces >> f) & 1u)) continue;
        double Zj[kNodePts];
#pragma unroll
        for (int j = 0; j < kNodePts; ++j) Zj[j] = 0.0;
#pragma unroll
        for (int el = 0; el < NEL; ++el) {
            const double *row = S + ((el * 2 + f) * kNodeMaxCells + c) * kNodePJ;
#pragma unroll
            for (int p = 0; p < kNodeTDeg; ++p) {
                const double ap = A_s[el][p];
#pragma unroll
                for (int j = 0; j < kNodePts; ++j) Zj[j] = fma(ap, row[p * kNodePts + j], Zj[j]);
            }
        }
#pragma unroll
        for (int i = 0; i < kNodePts; ++i) {
            double v = 0.0;
#pragma unroll
            for (int j = 0; j < kNodePts; ++j) v = fma(Lm_s[i * kNodePts + j], Zj[j], v);
            W[f][c][i] = v;
        }
    }
    __syncthreads();
    const double mu = a.mu[e];
    const double scale = 16.0 / 3.0 * kAlphaFs * kReCm2 / a.E_grid[e];
    const int warp = tid >> 5, lane = tid & 31;
    for (int d = warp; d < a.n_dir; d += kContractThreads / 32) {
        const double nz = a.n_hat[3 * d + 2];
        const int f = nz < 0.0 ? 0 : 1;
        const double lam = mu / fmax(fabs(nz), 1.0e-12);
        double acc = 0.0;
        for (int c = lane; c < nc; c += 32) {
#pragma unroll
            for (int i = 0; i < kNodePts; ++i) acc = fma(exp(-lam * nd_s[c * kNodePts + i]), W[f][c][i], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0 && acc != 0.0) atomicAdd(&a.spec[(int64_t)d * a.n_E + e], scale * acc);
    }
}

}  // namespace

cudaError_t launch_brem_node(const pb_brem_args &a, cudaStream_t s, int sms, const BremNodeHdr **hdr,
                             const int64_t **idx) {
    *hdr = nullptr;
    *idx = nullptr;
    if (a.work == nullptr || !brem_node_applies(a) || a.n_seg <= 0) return cudaSuccess;
    const BremNodeLayout l = brem_node_layout(a);
    if (a.work_bytes < (int64_t)l.total) return cudaSuccess;
    unsigned char *w = static_cast<unsigned char *>(a.work);
    BremNodeHdr *h = reinterpret_cast<BremNodeHdr *>(w + l.hdr);
    double *A = reinterpret_cast<double *>(w + l.A);
    double *S = reinterpret_cast<double *>(w + l.S);
    int64_t *ix = reinterpret_cast<int64_t *>(w + l.idx);
    cudaError_t err = cudaMemsetAsync(w, 0, l.zero_bytes, s);
    if (err != cudaSuccess) return err;
    brem_node_range_kernel<<<sms * 4, kNodeThreads, 0, s>>>(a, h);
    brem_node_setup_kernel<<<1, kNodeThreads, 0, s>>>(a, h);
    const int nq = a.n_E * a.n_el;
    brem_node_fit_kernel<<<(nq + 127) / 128, 128, 0, s>>>(a, h, A);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    using Accum = void (*)(const pb_brem_args, BremNodeHdr *, double *, int64_t *, int64_t);
    using Contract = void (*)(const pb_brem_args, const BremNodeHdr *, const double *, const double *);
    const Accum acc = a.n_el == 1 ? brem_node_accum_kernel<1> : brem_node_accum_kernel<2>;
    const Contract con = a.n_el == 1 ? brem_node_contract_kernel<1> : brem_node_contract_kernel<2>;
    const int smem = (int)node_accum_smem(a.n_el);
    err = cudaFuncSetAttribute(acc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return err;
    err = cudaFuncSetAttribute(acc, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (err != cudaSuccess) return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, acc, kNodeThreads, smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    acc<<<sms * per_sm, kNodeThreads, smem, s>>>(a, h, S, ix, l.cap);
    con<<<a.n_E, kContractThreads, 0, s>>>(a, h, A, S);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    *hdr = h;
    *idx = ix;
    return cudaSuccess;
}

}  // namespace pb
