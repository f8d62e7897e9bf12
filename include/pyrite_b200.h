/*
 * pyrite_b200 -- C ABI of the B200 (sm_100a) electron-transport and
 * radiation-scoring hot path of PyRITE.
 *
 * Every entry point takes plain C types: device pointers the caller owns,
 * sizes, and a CUDA stream passed as ``void *`` (NULL = the legacy default
 * stream). Calls are stream-ordered and return an int status (PB_OK = 0);
 * pb_last_error() returns the message of the calling thread's last failure.
 * Device-side conditions (a step limit reached, a queue overflow, a bounded
 * wait that gave up) are reported through the ``status`` word each call
 * writes, never by trapping. Nothing here allocates device memory unless
 * the function says so; workspace sizes are queried first.
 *
 * Reference interfaces replaced (paths relative to the PyRITE v0.36.2 tree):
 *   pb_transport      -- the per-electron transport core call
 *                        core((e_start, m, cap, keys), *core_args, scratch,
 *                        (seg_count, exit_code), ...)
 *                        src/pyrite/montecarlo/transport/batching.py:547-554,
 *                        kernels src/pyrite/montecarlo/transport/cores.py:96
 *                        (exact core) and lut.py:283 (LUT core); entry
 *                        sampling transport/beam_entry.py:23 and
 *                        transverse.py:197.
 *   pb_cxr_score      -- the incoherent PXR+CBS line scorer for a fixed
 *                        segment list, mc_cxr_spectrum
 *                        src/pyrite/montecarlo/spectrum/cxr/_spectrum.py:25,
 *                        batched route cxr/_batched.py:461-931.
 *   pb_brem_score     -- mc_brem_spectrum, Bethe-Heitler + Elwert
 *                        src/pyrite/montecarlo/spectrum/brem.py:829.
 *   pb_char_yields    -- the characteristic-line chunk kernel
 *                        src/pyrite/montecarlo/spectrum/_characteristic_chunk_kernel.py:120
 *                        and _accumulate_line_yields, characteristic.py:837;
 *   pb_char_spectrum  -- spec += line_yield * profile, characteristic.py:1219.
 *   pb_coherent_reduce -- the coherent (field-sum) CXR reduction of per-row
 *                        line records, cxr/_batched_finalize.py:209-243.
 *   pb_mlp_*          -- BF16 MLP surrogate of the reflection sum (no
 *                        counterpart in the reference; 6 -> 4x256 SiLU -> 512).
 */
#ifndef PYRITE_B200_H
#define PYRITE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB_ABI_VERSION 6

enum pb_status {
    PB_OK = 0,
    PB_ERR_INVALID = 1,   /* bad argument (size, pointer, enum) */
    PB_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    PB_ERR_UNSUPPORTED = 3,
    PB_ERR_CAPACITY = 4   /* an output buffer was too small (replay with more) */
};

/* Device status word bits (written by kernels, read by the host). */
enum pb_device_status {
    PB_DEV_STEP_LIMIT = 1u,      /* some history reached max_steps */
    PB_DEV_ROW_OVERFLOW = 2u,    /* rows beyond cap were counted, not stored */
    PB_DEV_QUEUE_OVERFLOW = 4u,  /* segment stream capacity exceeded */
    PB_DEV_WAIT_TIMEOUT = 8u,    /* a bounded wait gave up */
    PB_DEV_BAD_INPUT = 16u
};

enum pb_rng { PB_RNG_SPLITMIX = 0, PB_RNG_PHILOX = 1 };
enum pb_precision { PB_FP64 = 0, PB_MIXED = 1 };
enum pb_beam_mode { PB_BEAM_EXPLICIT = 0, PB_BEAM_SPOT = 1, PB_BEAM_TWISS = 2 };
enum pb_quadrature { PB_QUAD_NODE = 0, PB_QUAD_BINMEAN = 1 };
enum pb_elastic { PB_ELASTIC_SR = 0, PB_ELASTIC_ELSEPA = 2 };  /* the reference's elastic_model_code */

/* Exact analytic physics, padded per-layer element rows
 * (transport/batching.py:33-105). Device pointers. */
typedef struct pb_layers {
    int32_t n_layers;
    int32_t max_el;
    const double *z_top;         /* [n_layers] Angstrom */
    const double *z_bot;         /* [n_layers] */
    const int32_t *n_el;         /* [n_layers] */
    const double *J;             /* [n_layers*max_el] keV */
    const double *k;
    const double *coeff;
    const double *E_cross;
    const double *sr_rate_numer;
    const double *sr_joy_numer;
} pb_layers;

/* Uniform-log-energy LUT (transport/lut.py:64-283), packed by the host into
 * one 16-byte-aligned device buffer of ``elem_bytes``-sized values (8 for
 * FP64, 4 for the mixed path): [total_rate L x ne | dEds L x ne |
 * inv_beta ne | cdf L x max_el x ne | alpha L x max_el x ne], each block
 * starting at ``off_*`` values from ``base``. */
typedef struct pb_lut {
    int32_t n_energy;
    int32_t elem_bytes;
    double log_E_min;
    double inv_dlogE;
    const void *base;
    int64_t total_bytes;
    int64_t off_total_rate, off_dEds, off_inv_beta, off_cdf, off_alpha;
} pb_lut;

/* Entrance state (transport/beam_entry.py:23-160, transverse.py:197-226,
 * geometry.py:330-420). */
typedef struct pb_beam {
    int32_t mode;              /* pb_beam_mode */
    int32_t tilted;            /* nonzero: project spot onto the tilted face */
    double E0_keV;
    double beam_dir[3];        /* sample frame, unit */
    double e_x[3], e_y[3];     /* sample-frame lab spot axes */
    double basis[9];           /* beam frame basis, row-major, columns are axes */
    double sigma_x_ang, sigma_y_ang;  /* PB_BEAM_SPOT */
    double twiss_x[3], twiss_y[3];    /* PB_BEAM_TWISS: eps [mm rad], beta [mm/rad], alpha */
    uint64_t root;             /* counter-stream root of the entry draws */
    const double *pos0;        /* PB_BEAM_EXPLICIT: [n*3], [n*3], [n] device */
    const double *dir0;
    const double *E0;
} pb_beam;

/* Segment rows, slot i*cap + s, exactly as the reference core writes them. */
typedef struct pb_rows {
    double *r_mid;
    double *v_hat;
    double *L;
    double *E_start;
    double *E_end;
    double *t_start;
    double *t_end;
    int64_t *elec_id;
    int16_t *layer;
    int64_t *flight;
    int8_t *event;
} pb_rows;

/* Compact segment list: the scorers' input. SoA, device. */
typedef struct pb_segments {
    int64_t capacity;
    unsigned long long *count;  /* device counter (appended by pb_transport) */
    double *r_mid;    /* [capacity*3] */
    double *v_hat;    /* [capacity*3] */
    double *L;
    double *E_repr;   /* midpoint energy, keV */
    int64_t *elec_id;
    int32_t *layer;
} pb_segments;

/* Fused exit tallies (trajectory_summary.py:147-260): escaped primaries'
 * exit energy and polar exit angle to sample +z, uniform bins with explicit
 * underflow (index 0) and overflow (index n+1) slots, np.histogram edges. */
typedef struct pb_tallies {
    unsigned long long *fates;   /* [6] histories per exit code */
    unsigned long long *exit_E;  /* [n_E+2] */
    int32_t n_E;
    double E_lo, E_hi;
    unsigned long long *exit_theta;  /* [n_theta+2] */
    int32_t n_theta;
    double theta_lo, theta_hi;
    double *deposit;             /* [n_layers] keV lost continuously, per layer */
} pb_tallies;

/* ELSEPA tabulated elastic scattering (ABI 5), the reference's packed group
 * of src/pyrite/montecarlo/transport/scattering.py:398-490
 * (pack_elsepa_tables): every (layer, element) slot owns ``length`` energy
 * rows from ``start``; a row holds ln E, the log of the macroscopic rate
 * n sigma [1/cm], the piecewise-linear angular density in
 * mu = (1 - cos theta) / 2 on the shared grid ``mu``, its CDF and a guide
 * table of ``cells + 1`` panel bounds (cells a power of two). The rate is
 * interpolated log-log in energy (_elsepa_rate_scalar, :539-546) and a polar
 * cosine comes from one uniform inverted on both bracketing rows
 * (_sample_cos_theta_elsepa, :616-640). */
typedef struct pb_elsepa {
    int32_t n_mu;
    int32_t cells;
    const int64_t *start;      /* [n_layers * max_el] */
    const int64_t *length;     /* [n_layers * max_el], >= 2 for every element */
    const double *logE;        /* [rows] ln(E / eV), increasing within a slot */
    const double *log_rate;    /* [rows] */
    const double *cdf;         /* [rows * n_mu] */
    const double *pdf;         /* [rows * n_mu] */
    const double *mu;          /* [n_mu] */
    const int32_t *guide;      /* [rows * (cells + 1)] */
} pb_elsepa;

/* SBETHE table stopping (ABI 5), the reference's padded per-layer tables of
 * src/pyrite/montecarlo/transport/stopping.py:11-83 (prepare / pack): layer
 * L's first count[L] entries of row L hold ln(E / keV) and
 * ln(S / (keV/Angstrom)); the continuous stopping is their log-log
 * interpolation (_dEds_sbethe_scalar, :86-103), clamped at both ends. With
 * straggling each element's Urban mean is scaled by the table's stopping
 * over the spliced one (cores.py:595-604). count NULL keeps the spliced
 * Joy-Luo / Berger-Seltzer stopping. Exact core only (use_lut 0). */
typedef struct pb_stopping {
    int32_t width;
    const int32_t *count;      /* [n_layers], >= 2 */
    const double *logE;        /* [n_layers * width] */
    const double *logS;        /* [n_layers * width] */
} pb_stopping;

typedef struct pb_transport_args {
    int32_t rng;        /* pb_rng */
    int32_t precision;  /* pb_precision */
    int32_t use_lut;
    int32_t block_threads;  /* 0 = the default (256) */
    uint64_t seed;
    int64_t e_start;    /* first global history index */
    int64_t n;          /* histories */
    double E_cut_keV;
    int64_t max_steps;
    pb_layers layers;
    pb_lut lut;
    pb_beam beam;
    int64_t cap;            /* rows per history when rows.L != NULL */
    pb_rows rows;
    int64_t *seg_count;     /* [n] true row count (may exceed cap) */
    int8_t *exit_code;      /* [n] */
    double *final_pos;      /* [n*3] optional */
    double *final_dir;      /* [n*3] optional */
    double *final_E;        /* [n] optional */
    pb_segments seg;        /* optional compact stream */
    pb_tallies tallies;     /* optional (NULL pointers skip) */
    unsigned long long *work_counter;  /* device scratch, 1 word; zeroed by the call */
    unsigned int *status;   /* device status word (pb_device_status bits), OR-ed */
    /* ABI 4: Urban energy-loss straggling per flight (the reference's
     * straggling=True, transport/straggling.py with cores.py:654-700): each
     * flight's loss is sampled from the compound-Poisson Urban model of every
     * element of the layer instead of the deterministic midpoint loss.
     * Needs Z. Zero keeps the deterministic loss. */
    int32_t straggling;
    const double *Z;        /* [n_layers * max_el] atomic numbers */
    /* ABI 5: the elastic model, PB_ELASTIC_SR (the screened-Rutherford rates
     * and angles of pb_layers) or PB_ELASTIC_ELSEPA (the tables below; the
     * exact core only: use_lut must be 0, as the reference bypasses its LUT
     * for tabulated elastic scattering). */
    int32_t elastic_model;
    pb_elsepa elsepa;
    pb_stopping stopping;
} pb_transport_args;

/* CXR reflection rows and coupling tables (cxr/_batched.py:232-331). */
typedef struct pb_cxr_tables {
    int32_t n_g;
    const double *G;        /* [n_g*3] 1/Angstrom, sample frame */
    const double *ES;       /* [n_dir*n_g*3] sigma polarisation per direction */
    const double *EP;       /* [n_dir*n_g*3] pi polarisation per direction */
    const double *WM;       /* [n_g] */
    const int32_t *row_table;  /* [n_g] */
    int32_t n_tab;
    const double *E_tab;    /* [n_tab] eV, ascending */
    const double *chi_re;   /* [n_hkl*n_tab] */
    const double *chi_im;
    const double *u_re;
    const double *u_im;
    int32_t n_mu;
    const double *log_mu;   /* [n_mu*n_tab] */
    const double *delta;    /* [n_tab] */
    double lo_keep, hi_keep;
    /* Geometric E_tab (E_tab[i] = exp(tab_log0 + i tab_log_step)) enables a
     * closed-form bracket; tab_log_step <= 0 means a general ascending grid. */
    double tab_log0;
    double tab_log_step;
    /* Optional [n_tab]: max |delta| over E_tab[i:]. Bounds the refraction
     * shift of a root, so the mixed path can drop pairs that cannot reach
     * the keep window before solving for the root. */
    const double *delta_tail_absmax;
} pb_cxr_tables;

typedef struct pb_cxr_args {
    int32_t precision;      /* pb_precision */
    int32_t quadrature;     /* pb_quadrature; PB_QUAD_NODE needs the line buffer */
    int32_t n_dir;          /* detector directions (angular tiles) */
    const double *n_hat;    /* [n_dir*3] device */
    double thickness;
    int64_t Ne;             /* electrons counted (elec_id < Ne radiate) */
    int64_t n_seg;
    const double *r_mid, *v_hat, *L, *E_keV;  /* segment list (device) */
    const int64_t *elec_id;
    const unsigned long long *n_seg_device;  /* optional: read n_seg on device */
    pb_cxr_tables tables;
    int32_t n_E;            /* output nodes (node) or bins (bin-mean) */
    const double *E_grid;   /* [n_E] nodes */
    const double *edges;    /* [n_E+1] bin edges (bin-mean) */
    double exact_widths;    /* bin-mean: exact within this many widths; <=0: all exact */
    int32_t far_pad;        /* bin-mean, uniform axis: virtual centre bins each side
                               covering the keep window; -1 disables the far field */
    double *spec;           /* [n_dir*n_E] accumulated (+=), FP64, not normalised;
                               node quadrature: NULL keeps the lines only */
    double *far_moments;    /* workspace [n_dir*(n_E+2*far_pad)*3], zeroed by the call */
    /* Line buffer (node quadrature, and optional output of every kept line):
     * [line_capacity] each; direction index in line_dir. */
    int64_t line_capacity;
    unsigned long long *line_count;  /* device counter, zeroed by the call */
    double *line_E;
    double *line_a;
    double *line_w;
    int32_t *line_dir;
    /* Optional per-pair output for parity checks: [n_dir*n_seg*n_g] each. */
    double *pair_E;
    double *pair_a;
    double *pair_w;
    uint8_t *pair_good;
    unsigned int *status;
    /* Optional, with the line buffer: segment index of every kept line
     * (surrogate training targets are binned per (segment, direction)). */
    int64_t *line_seg;
    /* Layered absorber (cxr/_setup.py:1089 segment_escape_pieces with
     * layers, cxr/_batched.py:702-720). n_layer = 0 keeps the single slab
     * [0, thickness] and the log_mu escape rows. With 1 <= n_layer <= 4
     * contiguous planar layers [z_top[k], z_bot[k]) in depth order (thickness
     * = z_bot[n_layer-1]), each segment's escape is cut at the layer
     * boundaries it crosses and layer k attenuates with the piecewise-linear
     * mu_k(E) = mu_value[j] + (E - mu_knot[j]) mu_slope[j], 1/Angstrom at
     * the line energy E in eV, over its knots j in [mu_off[k], mu_off[k+1])
     * (j the last knot <= E, clipped to the table; 0 below the first knot),
     * as cxr/_escape_mu.py:41-57 evaluates a layer's composition. */
    int32_t n_layer;
    const double *z_top;    /* [n_layer] Angstrom */
    const double *z_bot;    /* [n_layer] */
    const int32_t *mu_off;  /* [n_layer + 1] */
    const double *mu_knot;  /* [mu_off[n_layer]] eV, ascending per layer */
    const double *mu_value;
    const double *mu_slope;
    /* Optional emitting-layer filter (cxr/_kernels.py:768-778, one crystal
     * layer of a stack per call): with seg_layer set, only segments whose
     * layer equals emit_layer radiate. */
    const int32_t *seg_layer;
    int32_t emit_layer;
    /* ABI 4, optional (NULL skips): work counters added to by the call,
     * [0] lines kept, [1] (line, bin) items deposited (bin-mean). */
    unsigned long long *counters;
} pb_cxr_args;

typedef struct pb_brem_args {
    int32_t precision;
    int32_t n_dir;
    const double *n_hat;    /* [n_dir*3] */
    double thickness;
    int64_t Ne;
    int64_t n_seg;
    const double *r_mid, *v_hat, *L, *E_keV;
    const int64_t *elec_id;
    const unsigned long long *n_seg_device;
    int32_t n_el;
    const double *Z;        /* [n_el] */
    const double *n_ang3;   /* [n_el] atoms / Angstrom^3 */
    int32_t n_E;
    const double *E_grid;   /* [n_E] eV */
    const double *mu;       /* [n_E] 1/Angstrom attenuation at the grid */
    double *spec;           /* [n_dir*n_E] accumulated (+=), not normalised */
    unsigned int *status;
    /* Layered absorber (brem.py:978-1005, 1195-1200): n_layer = 0 keeps the
     * single slab [0, thickness] with ``mu``; 1 <= n_layer <= 4 contiguous
     * planar layers [z_top[k], z_bot[k]) (thickness = z_bot[n_layer-1]),
     * each segment cut at the boundaries it crosses, layer k attenuating
     * with mu_layer[k][e] at grid energy e. */
    int32_t n_layer;
    const double *z_top;    /* [n_layer] Angstrom */
    const double *z_bot;    /* [n_layer] */
    const double *mu_layer; /* [n_layer*n_E] 1/Angstrom */
    /* Optional emitting-layer filter (emission.py:155-172: each layer
     * radiates with its own composition Z/n_ang3): with seg_layer set, only
     * segments whose layer equals emit_layer radiate. */
    const int32_t *seg_layer;
    int32_t emit_layer;
    /* Optional device workspace of the mixed single-slab path (bytes from
     * pb_brem_work_size; 16-byte aligned). With it the segments whose
     * electron energy lies in a narrow window below the batch's highest are
     * scored in the depth-node form (per-segment depth moments, then one
     * contraction per photon energy); the rest, or all of them where the
     * form does not apply, take the per-(segment, energy) form. NULL keeps
     * the per-(segment, energy) form throughout. */
    void *work;
    int64_t work_bytes;
} pb_brem_args;

/* Characteristic lines of one emitting element: per-segment shell
 * ionisation x cascade response x segment-mean escape transmission, summed
 * into line yields per direction. Tables are injected by the caller (the
 * reference's EEDL/EADL-derived inputs of _accumulate_line_yields). */
typedef struct pb_char_args {
    int32_t precision;      /* pb_precision: FP64, or MIXED (float escape exponentials) */
    int32_t n_dir;
    const double *n_hat;    /* [n_dir*3] */
    double thickness;       /* single slab [0, thickness] when n_layer == 0 */
    int32_t n_layer;        /* absorber layers (0: the single slab); <= 8 */
    const double *z_top;    /* [n_layer] Angstrom */
    const double *z_bot;    /* [n_layer] */
    int64_t Ne;             /* segments with elec_id < Ne emit */
    int64_t n_seg;
    const double *r_mid, *v_hat, *L, *E_keV;  /* segment list (device) */
    const int64_t *elec_id;
    const unsigned long long *n_seg_device;   /* optional: read n_seg on device */
    double n_atoms;         /* emitting number density, atoms / Angstrom^3 */
    int32_t n_shell;        /* ionised subshells, <= 40 */
    const double *shell_E;        /* packed per-shell projectile energies, eV, ascending per shell */
    const double *shell_sigma;    /* packed ionisation cross sections, cm^2 */
    const int64_t *shell_offset;  /* [n_shell+1] */
    int32_t n_line;         /* <= 256 */
    const double *response; /* [n_shell*n_line] photons per primary vacancy */
    const double *mu;       /* [max(n_layer,1)*n_line] attenuation at the line energies, 1/Angstrom */
    double *line_yield;     /* [n_dir*n_line] accumulated (+=), FP64: sum n L sigma_line T_escape */
    unsigned int *status;
    /* Optional emitting-layer filter: with seg_layer set, only segments whose
     * layer equals emit_layer emit (the element's own layer of a stack). */
    const int32_t *seg_layer;
    int32_t emit_layer;
} pb_char_args;

/* One GEMM of the BF16 MLP surrogate on tcgen05:
 *   D[M x N] = A[M x K] . B[N x K]^T   (bf16 in, FP32 accumulate)
 * then, per element: x = D + bias[n]; x *= silu'(dsilu_z[m][n]) when set;
 * out_f32[m][n] = x + beta out_f32[m][n]; h = act ? SiLU(x) : x;
 * out_bf16[m][n] = h; out_bf16_t[n][m] = h. Every output optional. */
typedef struct pb_mlp_gemm_args {
    int32_t M, N, K;          /* K a multiple of 16 */
    const void *A;            /* bf16 [M][lda], K contiguous */
    int64_t lda;
    const void *B;            /* bf16 [N][ldb], K contiguous */
    int64_t ldb;
    const float *bias;        /* [N] or NULL */
    int32_t act;              /* 0 identity, 1 SiLU */
    const float *dsilu_z;     /* [M][ldz] or NULL */
    int64_t ldz;
    float *out_f32;           /* [M][ldc] or NULL */
    int64_t ldc;
    float beta;
    void *out_bf16;           /* bf16 [M][ldh] or NULL */
    int64_t ldh;
    void *out_bf16_t;         /* bf16 [N][ldt] or NULL */
    int64_t ldt;
    unsigned int *status;     /* PB_DEV_WAIT_TIMEOUT if an MMA wait gave up */
} pb_mlp_gemm_args;

/* Surrogate inference: per (segment, direction) features
 *   x = (2 (ln E_MeV - ln E_lo)/(ln E_hi - ln E_lo) - 1, v.e_x / theta_max,
 *        v.e_y / theta_max, 2 clamp(z / thickness, 0, 1) - 1, u_d, v_d)
 * through 4 hidden layers of 256 SiLU units (bf16 weights, FP32 accumulate
 * on tcgen05); accumulates hsum[d][256] += L h4 and lsum[d] += L over the
 * segments with elec_id < Ne. The linear output layer is applied afterwards
 * by pb_mlp_head. Weights are pre-packed by pb_mlp_pack_umma. */
typedef struct pb_mlp_infer_args {
    int32_t n_dir;
    const float *dir_uv;      /* [n_dir][2] detector coordinates of each direction in [-1, 1] */
    double e_x[3], e_y[3];    /* transverse beam axes */
    double theta_max;         /* angle scale, rad */
    double E_lo_MeV, E_hi_MeV;
    double thickness;         /* Angstrom */
    int64_t Ne;
    int64_t n_seg;
    const double *r_mid, *v_hat, *L, *E_keV;
    const int64_t *elec_id;
    const unsigned long long *n_seg_device;
    const void *w1_packed;    /* pb_mlp_pack_umma(W1 [256][6..16], kc = 16): 8 KB */
    const void *w_packed[3];  /* pb_mlp_pack_umma(W2..W4 [256][256], kc = 64): 128 KB each */
    const float *bias[4];     /* b1..b4 [256] */
    double *hsum;             /* [n_dir][256] accumulated */
    double *lsum;             /* [n_dir] accumulated */
    unsigned int *status;
} pb_mlp_infer_args;

int pb_abi_version(void);
const char *pb_last_error(void);
int pb_device_count(int *count);

/* Transport: rows (parity replay), compact segments and/or fused tallies. */
int pb_transport(const pb_transport_args *args, void *stream);

/* Incoherent PXR + CBS lines of a segment list, reduced onto spectra. */
int pb_cxr_score(const pb_cxr_args *args, void *stream);

/* Bethe-Heitler + Elwert track-length bremsstrahlung of a segment list. */
int pb_brem_score(const pb_brem_args *args, void *stream);

/* Workspace bytes the depth-node form of pb_brem_score needs for these
 * arguments (precision, n_el, n_E, n_seg, n_layer): 0 where the form does
 * not apply (FP64, layered absorbers, more than two elements). */
int pb_brem_work_size(const pb_brem_args *args, int64_t *bytes);

/* Characteristic line yields of a segment list (accumulated). */
int pb_char_yields(const pb_char_args *args, void *stream);

/* spec[d][b] += sum_j line_yield[d][j] * profiles[j][b]: the yields spread
 * on the bins by per-eV line profiles (bin-integrated Lorentzians), before
 * the 1/(4 pi Ne) normalisation. All pointers device, FP64. */
int pb_char_spectrum(int32_t n_dir, int32_t n_line, int32_t n_E, const double *line_yield,
                     const double *profiles, double *spec, void *stream);

/* One whole pass of the hot path (ABI 5): zero the segment stream's count,
 * transport histories [transport.e_start, transport.e_start + transport.n)
 * into it, then score the stream with every CXR, bremsstrahlung and
 * characteristic argument set in order, all on ``stream`` -- the C form of
 * the reference's transport pass followed by its emission adapters
 * (montecarlo/transport/batching.py:547-554, then
 * montecarlo/runner/emission_adapters.py:53-112 per emission), which a
 * binding calls once per batch. The scorer sets read the segments through
 * their own pointers (normally transport.seg's arrays, with n_seg_device at
 * transport.seg.count). Every set is checked as its own entry point checks
 * it before anything is launched, so an argument error enqueues nothing; a
 * launch error part way returns with the earlier launches enqueued. */
typedef struct pb_transport_score_args {
    pb_transport_args transport;  /* transport.seg must be set */
    int32_t n_cxr;
    int32_t n_brem;
    int32_t n_char;
    int32_t pad_;
    const pb_cxr_args *cxr;       /* [n_cxr], host array */
    const pb_brem_args *brem;     /* [n_brem] */
    const pb_char_args *chars;    /* [n_char] */
} pb_transport_score_args;

int pb_transport_score(const pb_transport_score_args *args, void *stream);

/* Surrogate training: GEMM + fused epilogue (above). */
int pb_mlp_gemm(const pb_mlp_gemm_args *args, void *stream);
/* dY = g_scale (Y - t_scale T) (bf16, row-major [rows][cols] and transposed
 * [cols][ld_t]); *loss += sum (Y - t_scale T)^2. Y FP32 [rows][cols], T bf16 [rows][ldt_in]. */
int pb_mlp_mse_grad(int32_t rows, int32_t cols, const float *Y, const void *T, int64_t ldt_in, float t_scale,
                    float g_scale, void *dY, void *dYt, int64_t ld_t, float *loss, void *stream);
/* Group-aggregate loss gradient: rows in groups of S with normalised weights
 * w; per group and column A_hat = sum_s w_s Y_s, A = t_scale sum_s w_s T_s,
 * d = A_hat - A; *loss += sum d^2; dY_s = g_scale w_s d (bf16, row-major and
 * transposed [cols][ld_t]). */
int pb_mlp_group_mse_grad(int32_t groups, int32_t S, int32_t cols, const float *Y, const void *T, int64_t ldt_in,
                          const float *w, float t_scale, float g_scale, void *dY, void *dYt, int64_t ld_t,
                          float *loss, void *stream);
/* out[c] += sum_r X[r][c], X FP32 [rows][ld]. */
int pb_mlp_colsum(int32_t rows, int32_t cols, const float *X, int64_t ld, float *out, void *stream);
/* Adam (decoupled weight decay) on n packed FP32 parameters; bc1, bc2 the bias corrections. */
int pb_mlp_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                float wd, float bc1, float bc2, void *stream);
/* W FP32 [rows][cols] -> bf16 [rows][ldb] (zero padded) and, when Wt is set,
 * bf16 [pad_cols][ldt] transposed. */
int pb_mlp_pack(int32_t rows, int32_t cols, const float *W, void *Wb, int32_t ldb, void *Wt, int32_t ldt,
                int32_t pad_cols, void *stream);

/* Copy the segments of every stride-th history (elec_id % stride == 0) from
 * src into dst (dst->count zeroed by the call, then the number copied; beyond
 * dst->capacity the status word gets PB_DEV_QUEUE_OVERFLOW). src->count is
 * read on the device. */
int pb_segments_sample(const pb_segments *src, int64_t stride, const pb_segments *dst, unsigned int *status,
                       void *stream);

/* Copy n device byte ranges in one launch: desc (device memory) holds n
 * triples (source address, destination address, bytes) as int64. Ranges must
 * not overlap. The host API moves a step's scattered inputs and outputs
 * through one staging buffer each with it, so a step crosses the host link
 * in one copy each way. */
int pb_copy_segments(int32_t n, const int64_t *desc, void *stream);

/* Surrogate inference (above). */
int pb_mlp_infer(const pb_mlp_infer_args *args, void *stream);
/* The inference kernel's inputs as a matrix, for training: X bf16
 * [n_dir * n_seg][16] (row d * n_seg + s) and weight [n_dir * n_seg]. */
int pb_mlp_features(const pb_mlp_infer_args *args, void *X, float *weight, void *stream);
/* spec[d][o] += t_scale (W5[o] . hsum[d] + b5[o] lsum[d]); W5 FP32 [n_out][256]. */
int pb_mlp_head(int32_t n_dir, int32_t n_out, const float *W5, const float *b5, const double *hsum,
                const double *lsum, double t_scale, double *spec, void *stream);
/* W FP32 [256][cols] -> bf16 chunks of kc (16, 32 or 64) columns in the
 * interleaved core-matrix layout the inference kernel streams. */
int pb_mlp_pack_umma(int32_t cols, int32_t kc, const float *W, void *out, void *stream);

/* Bin a line buffer per (segment, direction) pair onto a uniform coarse
 * grid: target[(line_dir - dir0) * n_seg + line_seg][b] += w (pi / a) m_b /
 * width, m_b the line's exact sinc^2 mass in bin b (float antiderivatives,
 * bins within 64 first-zero widths and 64 bins of the centre). Lines whose
 * direction falls outside [dir0, dir0 + n_dir_chunk) are skipped. */
int pb_cxr_bin_lines(int64_t n_lines, const double *line_E, const double *line_a, const double *line_w,
                     const int32_t *line_dir, const int64_t *line_seg, int32_t dir0, int32_t n_dir_chunk,
                     int64_t n_seg, double lo_eV, double width_eV, int32_t n_bins, float *target, void *stream);

/* Coherent route, record prologue: the per-row line records of
 * pb_coherent_reduce from a segment list, for one detector direction
 * (cxr.n_dir = 1), FP64, single slab. Replaces the reference's record
 * building of cxr/_batched.py:561-660 (the complex PXR+CBS amplitude per
 * polarisation of cxr/_batched.py:600-625, escape-piece ends and formation
 * coefficients of cxr/_formation.py:58-81 and cxr/_batched.py:627-633, the
 * exact vacuum centre, width and recoil phase over the electron's age of
 * cxr/_recoil.py:118-147, the phase terms of cxr/_setup.py:1023-1026). Row g
 * (a reflection x mosaic orientation, the row of cxr.tables) holds its kept
 * pairs in segment order; rows follow one another (row_off[g] ..
 * row_off[g+1], written by the call). Kept pairs past ``capacity`` are
 * dropped and set PB_DEV_QUEUE_OVERFLOW. ``t_start`` holds each segment's
 * start age [Angstrom] (NULL = 0). cxr.quadrature, the spectrum and line
 * buffer fields are not read. */
typedef struct pb_coherent_records_args {
    pb_cxr_args cxr;           /* segments, direction, tables (n_dir = 1) */
    const double *t_start;     /* [n_seg] or NULL */
    int64_t capacity;          /* records each output array holds */
    double *E_vac, *a_vac, *phase_slope, *g_phase, *cs_re, *cs_im, *cp_re, *cp_im, *L_esc, *half_dL, *apb,
        *bma, *q;              /* [capacity] */
    int64_t *row_off;          /* [n_g + 1] out */
    void *work;                /* pb_coherent_records_work_size bytes, 256-byte aligned */
    uint64_t work_bytes;
    unsigned int *status;      /* device status word, OR-ed (NULL: not reported) */
    int64_t *elec_out;         /* ABI 5, optional [capacity]: each record's electron (the
                                  segment's elec_id), for the decoherence blend */
} pb_coherent_records_args;

int pb_coherent_records_work_size(int64_t n_seg, int32_t n_g, uint64_t *bytes);
int pb_coherent_records(const pb_coherent_records_args *args, void *stream);

/* pb_cxr_score without any device allocation, for callers that cannot call
 * cudaMalloc: code running inside an allocator or memory-pool callback, an
 * embedding runtime that owns all device memory, or a deployment that fixes
 * every allocation at load time. No counterpart in the reference.
 *
 * Bin-mean quadrature only. ``far_moments`` is ignored: the far-field
 * workspace is a fixed device array built into the library (2 MiB per GPU
 * that loads it, held until the process exits), limited to
 * n_dir * (n_E + 2 far_pad) * 3 <= 262144 FP64 moments; larger requests
 * fail with PB_ERR_CAPACITY. The caller still owns every input and output.
 * The arguments are checked as pb_cxr_score checks them (same error codes),
 * except that far_moments may be NULL.
 * The first call in a CUDA context resolves the array's device address
 * (cudaGetSymbolAddress) and caches it under the context's ID, so make that
 * first call before any stream capture; a context created later (after
 * cudaDeviceReset, or by the driver API) gets its own lookup on its first
 * call. All calls share the one array and clear it on entry: calls that
 * overlap on the GPU (different streams, threads or processes sharing a
 * context) race on it and must be serialised by the caller. */
int pb_cxr_score_noalloc(const pb_cxr_args *args, void *stream);

/* Coherent (field-sum) CXR reduction of per-row line records: for every row
 * r (one reflection x mosaic orientation) and output energy E_k,
 *   F_pol(E) = sum_j c_pol,j F_j(E) exp(i phi_j(E)),  pol = sigma, pi,
 *   phi_j(E) = phase_slope_j E - g_phase_j - L_esc,j delta_omega(E),
 *   F_j(E)   = formation factor of v = a_vac_j (E - E_vac_j) - half_dL_j
 *              delta_omega(E) with (apb_j, bma_j, q_j),
 *   spec[k] += scale * sum_r row_weight[r] (|F_sigma|^2 + |F_pi|^2).
 * Rows add incoherently; lines inside a row keep their phase. Replaces the
 * per-row reduction of the reference's coherent route,
 * src/pyrite/montecarlo/spectrum/cxr/_batched_finalize.py:209-243 and its
 * CUDA form run_coherent_reduction_kernel
 * (src/pyrite/montecarlo/spectrum/coherent_jit_kernel.py), formation factor
 * cxr/_formation.py:84-130; the record fields are the ``per_cxr`` tuple of
 * cxr/_batched.py:646-660, laid out row after row (row r holds lines
 * row_off[r] .. row_off[r+1]). Phases are evaluated in FP64 and reduced to
 * [-pi, pi] before FP32 sin/cos; per-chunk fields are FP32 and the row sums
 * FP64, in a fixed order (the result does not depend on the launch). */
typedef struct pb_coherent_args {
    int32_t n_row;
    int32_t n_E;
    int64_t n_line;                 /* == row_off[n_row] */
    const int64_t *row_off;         /* [n_row + 1], nondecreasing, row_off[0] = 0 */
    const double *row_weight;       /* [n_row] */
    const double *E;                /* [n_E] photon energies, eV */
    const double *delta_omega;      /* [n_E] delta(E) omega(E), 1/Angstrom */
    const double *E_vac, *a_vac, *phase_slope, *g_phase;   /* [n_line] each */
    const double *cs_re, *cs_im, *cp_re, *cp_im;
    const double *L_esc, *half_dL, *apb, *bma, *q;
    double scale;                   /* e.g. 1 / electrons */
    double sinc_cutoff;             /* > 0: a line adds nothing where |v| > sinc_cutoff
                                       (coherent_jit_kernel.py:752-760); 0 = no window */
    double *spec;                   /* [n_E], accumulated into */
    void *work;                     /* pb_coherent_work_size bytes, 256-byte aligned */
    uint64_t work_bytes;
    unsigned int *status;           /* optional device word: PB_DEV_BAD_INPUT when row_off
                                       is not a partition of [0, n_line) (rows are then
                                       clamped into it) */
} pb_coherent_args;

/* Workspace bytes pb_coherent_reduce needs for these sizes. */
int pb_coherent_work_size(int32_t n_row, int64_t n_line, int32_t n_E, uint64_t *bytes);
int pb_coherent_reduce(const pb_coherent_args *args, void *stream);

/* The sampled-bunch decoherence factor of every row,
 *   F[r, k] = |(1/n_pop) sum_p exp(i (omega_k A_p - (G_r,x x0_p + G_r,y y0_p)))|^2,
 * A_p = t0_p - n_perp . xy0_p the population's emission-time offsets
 * (Angstrom) and xy0_p its transverse entry offsets, FP64 throughout.
 * Replaces the reference's row factor, src/pyrite/montecarlo/spectrum/cxr/
 * _per_hkl.py:121-160 with the population of cxr/_setup.py:745-760. */
typedef struct pb_decoherence_args {
    int32_t n_row;
    int32_t n_pop;
    int32_t n_E;
    int32_t pad_;
    const double *G;         /* [n_row * 3] reciprocal vectors of the rows (x, y used) */
    const double *A_pop;     /* [n_pop] */
    const double *xy0_pop;   /* [n_pop * 2] */
    const double *omega;     /* [n_E] omega(E) = E / (hbar c), 1/Angstrom */
    double *F;               /* [n_row * n_E], written */
} pb_decoherence_args;

int pb_decoherence_factor(const pb_decoherence_args *args, void *stream);

/* The coherent reduction with the sampled-bunch decoherence blend: every row
 * mixes its all-electron field (flat) and the sum over electrons of each
 * electron's own squared field (grouped) by the row factor F,
 *   spec[k] += scale * sum_r row_weight[r] (F[r,k] flat_r(E_k)
 *                                           + (1 - F[r,k]) grouped_r(E_k)).
 * Replaces src/pyrite/montecarlo/spectrum/cxr/_batched_finalize.py:163-243
 * (_decoherence_blend with every energy kept) and its per-electron grouped
 * row (cxr/_per_hkl.py:457-500). A row's lines of one electron must be
 * contiguous, electrons in nondecreasing id order (the record prologue's
 * segment order); a decrease sets PB_DEV_BAD_INPUT in base.status. The
 * flat and grouped sums come out of one pass over the lines. */
typedef struct pb_coherent_blend_args {
    pb_coherent_args base;   /* base.work: pb_coherent_blend_work_size bytes */
    const int64_t *elec_id;  /* [n_line] emitting electron of every line */
    const double *F_row;     /* [n_row * n_E] row factors (pb_decoherence_factor) */
} pb_coherent_blend_args;

int pb_coherent_blend_work_size(int32_t n_row, int64_t n_line, int32_t n_E, uint64_t *bytes);
int pb_coherent_blend(const pb_coherent_blend_args *args, void *stream);

/* Streamed coherent reduction (ABI 5), the reference's field-plane route
 * (src/pyrite/montecarlo/spectrum/coherent_stream_jit_kernel.py): a row's
 * complex field must be summed over every segment before it is squared, so
 * block after block of records (pb_coherent_records of one segment block)
 * is folded into persistent FP64 field planes fields[n_row][4][n_E]
 * (sigma re, sigma im, pi re, pi im), and with elec_id the per-electron
 * squared fields into power[n_row][n_E] (a block must then end on an
 * electron boundary). pb_coherent_finalize squares and weights them:
 *   spec[k] += scale * sum_r row_weight[r] (F[r,k] |field_r(E_k)|^2
 *                                           + (1 - F[r,k]) power_r(E_k)),
 * F = 1 (no power needed) when F_row is NULL. base.spec is unused by the
 * accumulation; base.work is pb_coherent_blend_work_size bytes with elec_id,
 * pb_coherent_work_size bytes without. Each cell has one writer per launch:
 * no atomics, results independent of the launch. */
typedef struct pb_coherent_stream_args {
    pb_coherent_args base;
    const int64_t *elec_id;  /* optional [n_line] */
    double *fields;          /* [n_row * 4 * n_E], accumulated */
    double *power;           /* [n_row * n_E], accumulated when elec_id is set */
} pb_coherent_stream_args;

int pb_coherent_accumulate(const pb_coherent_stream_args *args, void *stream);
int pb_coherent_finalize(int32_t n_row, int32_t n_E, const double *row_weight, const double *fields,
                         const double *power, const double *F_row, double scale, double *spec, void *stream);

#ifdef __cplusplus
}
#endif
#endif
