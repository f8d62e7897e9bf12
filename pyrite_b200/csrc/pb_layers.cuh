// Escape geometry of a planar layered absorber, shared by the CXR and
// bremsstrahlung scorers.
//
// A photon emitted at depth z leaves along n_hat through the layers between
// z and the face it exits by (the entrance face when n_z < 0, the back face
// otherwise); the path it runs in layer k is the z-extent it crosses there
// divided by |n_z| (segment_escape.py:63-70, attenuation.py:270-277).
// Within one layer m these extents are affine in z: on the entrance side the
// layers above m are crossed whole and m for z - z_top[m]; on the back side m
// for z_bot[m] - z and the layers below whole. So with C_up[m] = sum_{k<m}
// mu_k t_k and C_dn[m] = sum_{k>m} mu_k t_k the optical depth is
//     tau = (C_side[m] + mu_m w) / |n_z|,  w = z - z_top[m] or z_bot[m] - z.
// A segment is cut where it crosses a layer boundary (segment_escape.py:
// 217-222, 246-263: cuts at the tops of layers 1..n-1, pieces shorter than
// 1e-12 of the segment dropped), each piece is affine, and its segment-mean
// transmission is the closed form of mean_transmission over its end depths.
#pragma once

#include <stdint.h>

namespace pb {

constexpr int kMaxEscLayers = 4;

// One affine piece of a segment: its share of the segment's length and the
// depth below the top of its layer m at both ends (clamped to the layer).
struct EscPiece {
    double f;
    double u0, u1;
    int m;
};

// _cut_at_zero (segment_escape.py:134-140): the fraction where an affine
// quantity changes sign, or 1 if it does not inside (0, 1).
__host__ __device__ inline double esc_cut_at_zero(double start, double end) {
    const double den = start - end;
    const double fr = start / (den == 0.0 ? 1.0 : den);
    return (fr > 0.0 && fr < 1.0) ? fr : 1.0;
}

// Split the segment from depth z0 to z1 at the layer boundaries; returns the
// number of pieces (<= n_layer) written to ``out``, in order along the
// segment. Layers are contiguous: z_bot[k] == z_top[k + 1].
__host__ __device__ inline int esc_pieces(double z0, double z1, int n_layer, const double *z_top,
                                          const double *z_bot, EscPiece *out) {
    double cuts[kMaxEscLayers + 1];
    int nc = 0;
    cuts[nc++] = 0.0;
    for (int k = 1; k < n_layer; ++k) cuts[nc++] = esc_cut_at_zero(z0 - z_top[k], z1 - z_top[k]);
    cuts[nc++] = 1.0;
    // insertion sort (at most kMaxEscLayers + 1 entries)
    for (int i = 1; i < nc; ++i) {
        const double v = cuts[i];
        int j = i - 1;
        while (j >= 0 && cuts[j] > v) {
            cuts[j + 1] = cuts[j];
            --j;
        }
        cuts[j + 1] = v;
    }
    int np = 0;
    const double dz = z1 - z0;
    for (int i = 0; i + 1 < nc; ++i) {
        const double w = cuts[i + 1] - cuts[i];
        if (!(w > 1.0e-12)) continue;
        const double za = z0 + cuts[i] * dz;
        const double zb = z0 + cuts[i + 1] * dz;
        const double zm = 0.5 * (za + zb);
        int m = 0;
        while (m + 1 < n_layer && zm >= z_top[m + 1]) ++m;
        const double t = z_bot[m] - z_top[m];
        const double ua = za - z_top[m], ub = zb - z_top[m];
        EscPiece p;
        p.f = w;
        p.u0 = ua < 0.0 ? 0.0 : (ua > t ? t : ua);
        p.u1 = ub < 0.0 ? 0.0 : (ub > t ? t : ub);
        p.m = m;
        if (np < kMaxEscLayers) out[np] = p;
        ++np;
    }
    return np < kMaxEscLayers ? np : kMaxEscLayers;
}

// ExactMuTable.__call__ (cxr/_escape_mu.py:49-57): piecewise-linear mu(E) on
// the knots [0, n): j = searchsorted(knots, E, "right") - 1 clipped to the
// table, 0 below the first knot.
__device__ __forceinline__ double esc_mu_at(const double *knot, const double *value, const double *slope, int n,
                                            double E) {
    if (n <= 0 || !(E >= knot[0])) return 0.0;
    int lo = 0, hi = n;  // first index with knot > E lies in [lo, hi]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (knot[mid] <= E) lo = mid + 1;
        else hi = mid;
    }
    int j = lo - 1;
    if (j < 0) j = 0;
    if (j > n - 1) j = n - 1;
    return value[j] + (E - knot[j]) * slope[j];
}

// v[m] for m in [0, kMaxEscLayers) without a local-memory array.
template <class Real>
__device__ __forceinline__ Real esc_pick(const Real (&v)[kMaxEscLayers], int m) {
    Real r = v[0];
#pragma unroll
    for (int k = 1; k < kMaxEscLayers; ++k)
        if (m == k) r = v[k];
    return r;
}

}  // namespace pb
