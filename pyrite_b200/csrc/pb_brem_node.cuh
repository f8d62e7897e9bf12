// Depth-node form of the mixed single-slab bremsstrahlung scorer: state
// shared between its kernels (pb_brem_node.cu) and the per-(segment, energy)
// kernels that score the segments it leaves out (pb_brem.cu).
#pragma once

#include <cstdint>

#include "pb_internal.h"

namespace pb {

constexpr int kNodeMaxCells = 64;   // depth cells of the escape interpolation
constexpr int kNodePts = 8;         // Chebyshev nodes per cell (degree 7)
constexpr int kNodeTDeg = 6;        // coefficients of the electron-energy polynomial (degree 5)
constexpr int kNodePJ = kNodeTDeg * kNodePts;  // moments per (element, face, cell)
constexpr int kNodeMaxEl = 2;       // elements the shared accumulator holds
constexpr double kNodeWindow = 1.1; // T_hi / T_lo of the energy window at most
constexpr double kNodeTip = 2.5;    // T_lo >= 2.5 k_max: the window stays clear of the spectrum's tip
constexpr int kNodeUniform = 5;     // cells of width h_min before the geometric growth
constexpr double kNodeGrowth = 1.2;  // deeper cells: width a fifth of their start depth

// Launch state in the caller's workspace (zeroed before each launch).
struct BremNodeHdr {
    unsigned long long t_max_bits;   // atomicMax of T over radiating segments (bits of a non-negative double)
    unsigned long long t_minc_bits;  // atomicMax of ~bits: the smallest T
    unsigned long long n_out;        // segments left to the per-(segment, energy) form
    unsigned int ok;                 // the node form scores this launch
    unsigned int faces;              // bit 0: a direction leaves through the top face, bit 1: the bottom
    int n_cells;
    int pad_;
    double T_lo, T_hi, Tc, Th;       // electron-energy window [T_lo, T_hi], centre and half-width
    double h_min, z_g;               // uniform cell width and the depth where the growth starts
    double zb[kNodeMaxCells + 1];    // cell boundaries, depth below the exit face
    double node[kNodeMaxCells * kNodePts];
    double Lm[kNodePts * kNodePts];  // Lagrange basis of the cell nodes in monomials of t: [i][j]
};

// Byte offsets of the workspace parts.
struct BremNodeLayout {
    size_t hdr, A, S, idx, total, zero_bytes;
    int64_t cap;  // capacity of the left-out segment list
};

__host__ __device__ inline BremNodeLayout brem_node_layout(const pb_brem_args &a) {
    BremNodeLayout l;
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    l.hdr = 0;
    l.A = up(sizeof(BremNodeHdr));
    l.S = up(l.A + sizeof(double) * (size_t)a.n_E * (size_t)a.n_el * kNodeTDeg);
    l.idx = up(l.S + sizeof(double) * (size_t)a.n_el * 2 * kNodeMaxCells * kNodePJ);
    l.cap = a.n_seg / 8 + 4096;
    l.total = l.idx + sizeof(int64_t) * (size_t)l.cap;
    l.zero_bytes = l.idx;  // header, coefficients and moments
    return l;
}

// Whether the node form can take these arguments at all (the device then
// decides per launch from the segments and the directions).
__host__ __device__ inline bool brem_node_applies(const pb_brem_args &a) {
    return a.precision == PB_MIXED && a.n_layer == 0 && a.n_el >= 1 && a.n_el <= kNodeMaxEl && a.n_E >= 1;
}

// Runs the node form's kernels when the workspace is set; *hdr and *idx then
// point at the launch state and the left-out segment list the
// per-(segment, energy) kernels read, else they are null.
cudaError_t launch_brem_node(const pb_brem_args &a, cudaStream_t s, int sms, const BremNodeHdr **hdr,
                             const int64_t **idx);

}  // namespace pb
