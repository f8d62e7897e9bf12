/*
 * CPU ORACLE -- test infrastructure, never the product.
 *
 * C restatement of the reference's transport and emission-scoring arithmetic
 * (PyRITE v0.36.2). Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline call into it, always as the checker or the timed CPU reference,
 * never as the product path.
 */
#ifndef PYRITE_ORACLE_H
#define PYRITE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_RNG_SPLITMIX = 0, OR_RNG_PHILOX = 1 };

/* Exit codes: src/pyrite/montecarlo/transport/cores.py:88-93 */
enum {
    OR_EXIT_CUTOFF = 0,
    OR_EXIT_BACKSCATTERED = 1,
    OR_EXIT_TRANSMITTED = 2,
    OR_EXIT_SIDE = 3,
    OR_EXIT_STEP_LIMITED = 4,
    OR_EXIT_NOT_ENTERED = 5
};

/* Row events: src/pyrite/montecarlo/transport/events.py:35-42 */
enum {
    OR_EVENT_ELASTIC = 0,
    OR_EVENT_LAYER_BOUNDARY = 2,
    OR_EVENT_EXIT_TOP = 4,
    OR_EVENT_EXIT_BOTTOM = 5,
    OR_EVENT_CUTOFF = 7
};

/* ELSEPA tabulated elastic group (scattering.py:398-490, pack_elsepa_tables):
 * per (layer, element) a run of energy rows, each an angular density on the
 * shared mu grid with its CDF and guide table. */
typedef struct {
    int n_mu;
    int cells;                   /* guide cells (a power of two) */
    const int64_t *start;        /* [n_layers*max_el] first row */
    const int64_t *length;       /* [n_layers*max_el] rows */
    const double *logE;          /* [rows] ln(E / eV) */
    const double *log_rate;      /* [rows] ln(n sigma / cm^-1) */
    const double *cdf;           /* [rows*n_mu] */
    const double *pdf;           /* [rows*n_mu] */
    const double *mu;            /* [n_mu] */
    const int32_t *guide;        /* [rows*(cells+1)] */
} or_elsepa;

double or_elsepa_rate(const or_elsepa *t, int64_t start, int64_t length, double E_keV);
double or_elsepa_cos_theta(const or_elsepa *t, int64_t start, int64_t length, double E_keV, double xi);

/* Padded per-layer element tables: batching.py:33-105 (pack_layer_tables). */
typedef struct {
    int n_layers;
    int max_el;
    const double *z_top;         /* [n_layers] Angstrom */
    const double *z_bot;         /* [n_layers] */
    const int *n_el;             /* [n_layers] */
    const double *J;             /* [n_layers*max_el] keV */
    const double *k;             /* Joy-Luo k */
    const double *coeff;         /* (n_i / 0.602214076) Z */
    const double *E_cross;       /* Joy-Luo / Berger-Seltzer crossover, keV */
    const double *sr_rate_numer; /* 5.21e-21 Z^2 4 pi n_cm3 */
    const double *sr_joy_numer;  /* 3.4e-3 Z^0.67 */
    const double *Z;             /* [n_layers*max_el] atomic numbers (Urban straggling) */
    int straggling;              /* 1: Urban energy-loss straggling per flight */
    const or_elsepa *elsepa;     /* non-NULL: ELSEPA elastic model (elastic_model_code 2) */
    /* SBETHE table stopping (stopping.py:11-103): per layer sb_count[L]
     * nodes of ln(E / keV) and ln(S / (keV/Angstrom)); sb_count NULL keeps
     * the spliced analytic stopping. */
    int sb_width;
    const int *sb_count;
    const double *sb_logE;
    const double *sb_logS;
} or_layers;

double or_sbethe_dEds(const or_layers *ly, int L, double E);

/* Urban energy-loss straggling (straggling.py:37-333). */
double or_dEds_element(double J, double k, double coeff, double E_cross, double E);
double or_urban_sample_element(double Z, double J, double C, double E, double s, uint64_t key,
                               uint64_t *counter);
void or_urban_moments_element(double Z, double J, double C, double E, double s, double *mean, double *var);

/* Segment rows, slot i*cap + s (cores.py:911-935). */
typedef struct {
    double *r_mid;   /* [rows*3] */
    double *v_hat;   /* [rows*3] */
    double *L;
    double *E_start;
    double *E_end;
    double *t_start;
    double *t_end;
    int64_t *elec_id;
    int16_t *layer;
    int64_t *flight;
    int8_t *event;
} or_rows;

uint64_t or_splitmix64(uint64_t x);
uint64_t or_stream_key(uint64_t seed, uint64_t elec);
double or_stream_uniform(uint64_t key, uint64_t counter);
void or_philox4x32_10(uint32_t ctr[4], uint32_t key[2]);
double or_philox_uniform(uint64_t key, uint64_t draw);

double or_beta_from_keV(double E);
double or_dEds_spliced(const or_layers *ly, int L, double E);
double or_sr_rate(double E, double sr_rate_numer, double sr_joy_numer);
double or_cos_theta_sr(double alpha, double R);
void or_rotate(double *dx, double *dy, double *dz, double cos_t, double phi);

void or_transport(const or_layers *ly, int rng_kind, uint64_t seed, int64_t e_start, int64_t n,
                  double E_cut, int64_t max_steps, int64_t cap, double *pos, double *dir, double *E,
                  double *clock, or_rows *rows, int64_t *seg_count, int8_t *exit_code,
                  int n_threads);

/* Uniform-log-energy transport LUT (src/pyrite/montecarlo/transport/lut.py:64-283). */
typedef struct {
    int n_layers;
    int max_el;
    int n_energy;
    double log_E_min;
    double inv_dlogE;
    const double *z_top;      /* [n_layers] */
    const double *z_bot;
    const int *n_el;
    const double *total_rate; /* [n_layers*n_energy] 1/cm */
    const double *dEds;       /* [n_layers*n_energy] keV/Angstrom */
    const double *inv_beta;   /* [n_energy] */
    const double *cdf;        /* [n_layers*max_el*n_energy] */
    const double *alpha;      /* [n_layers*max_el*n_energy] */
} or_lut;

void or_transport_lut(const or_lut *t, int rng_kind, uint64_t seed, int64_t e_start, int64_t n,
                      double E_cut, int64_t max_steps, int64_t cap, double *pos, double *dir,
                      double *E, double *clock, or_rows *rows, int64_t *seg_count,
                      int8_t *exit_code);

/* ---- CXR line chain (PXR + CBS, incoherent, single slab) ---------------- */
typedef struct {
    int n_g;           /* reflection x orientation rows */
    const double *G;   /* [n_g*3] sample-frame reciprocal vectors, 1/Angstrom */
    const double *ES;  /* [n_g*3] sigma polarization */
    const double *EP;  /* [n_g*3] pi polarization */
    const double *WM;  /* [n_g] mosaic weight */
    const int *row_table; /* [n_g] coupling-table row */
    int n_tab;
    const double *E_tab;  /* [n_tab] eV */
    const double *chi_re; /* [n_hkl*n_tab] */
    const double *chi_im;
    const double *u_re;   /* U_g / m_e c^2 */
    const double *u_im;
    int n_mu;
    const double *log_mu; /* [n_mu*n_tab] log(1/Angstrom) per absorber element */
    const double *delta;  /* [n_tab] 1 - Re n */
    double lo_keep, hi_keep;
} or_cxr_tables;

/* Planar layered absorber (segment_escape.py:193-272): layers [z_top, z_bot)
 * in depth order; mu_off/mu_knot/mu_value/mu_slope give each layer's exact
 * piecewise-linear mu(E) (cxr/_escape_mu.py:41-57), used by the CXR chain. */
typedef struct {
    int n_layer;
    const double *z_top, *z_bot;
    const int *mu_off;
    const double *mu_knot, *mu_value, *mu_slope;
} or_layer_escape;

typedef struct {
    double n_hat[3];
    double thickness;  /* Angstrom; slab 0 <= z <= thickness (stack: its total) */
    const or_layer_escape *layers;  /* NULL: the single slab */
} or_cxr_geom;

/* One line per (segment, row): E_res [eV], a_width [1/eV], weight; good = 0
 * when the pair is dropped. Arrays are [n_seg*n_g], segment-major. */
void or_cxr_lines(const or_cxr_tables *t, const or_cxr_geom *geo, int64_t n_seg,
                  const double *v_hat, const double *E_keV, const double *L_ang,
                  const double *r_mid, const int64_t *elec_id, int64_t Ne, double *E_res,
                  double *a_width, double *weight, uint8_t *good, int n_threads);

/* Coherent route line records per (segment, row), single slab, one escape
 * piece per segment (cxr/_batched.py:561-660 on the rows of _batched_block,
 * cxr/_batched.py:479-559): rec[k][s*n_g + g] for the 13 fields
 * E_vac, a_vac, phase_slope, g_phase, cs_re, cs_im, cp_re, cp_im, L_esc,
 * half_dL, apb, bma, q; good = 0 where the reference drops the pair.
 * t_ang: segment start ages [Angstrom] (NULL = 0). */
#define OR_COH_FIELDS 13
void or_cxr_coherent_records(const or_cxr_tables *t, const or_cxr_geom *geo, int64_t n_seg,
                             const double *v_hat, const double *E_keV, const double *L_ang,
                             const double *r_mid, const double *t_ang, const int64_t *elec_id,
                             int64_t Ne, double *const rec[OR_COH_FIELDS], uint8_t *good);

/* spec[e] += sum_j w_j sinc^2(a_j (E_e - E_j)/pi) (cxr/_cpu_reduce.py:26-50) */
void or_reduce_node(int64_t n_lines, const double *E_res, const double *a_width,
                    const double *weight, int64_t n_e, const double *E_grid, double *spec,
                    int n_threads);

/* spec[b] += sum_j w_j (1/width_b) int_bin sinc^2 (exact, Si based) */
void or_reduce_binmean(int64_t n_lines, const double *E_res, const double *a_width,
                       const double *weight, int64_t n_bins, const double *edges, double *spec,
                       int n_threads);

double or_sincsq_tail(double x);
double or_si_minus_half_pi(double t);

/* mean of exp(-tau) between linear end depths (segment_escape.py:276-289) */
double or_mean_transmission(double tau0, double tau1);

/* exact second-order PXR numerator and CBS factor (cxr/_recoil.py:35-76) */
void or_quantum_line_factors(double h, double gamma, double vdg, double k_dot_v, double k_dot_g,
                             double g2, double k2, double v_dot_e, double g_dot_e, double k_dot_e,
                             double *pxr_num, double *f_cbs);

/* ---- Bethe-Heitler + Elwert bremsstrahlung (spectrum/brem.py:431-505) --- */
void or_brem_spectrum(int64_t n_seg, const double *E_keV, const double *L_ang,
                      const double *r_mid, const double *v_hat, int n_el, const double *Z,
                      const double *n_cm3, double thickness, const double n_hat[3], int64_t n_e,
                      const double *E_grid, const double *mu_grid, double *spec, int n_threads);

/* Layered bremsstrahlung (brem.py:978-1005,1195-1239): segments cut into
 * escape pieces, each piece attenuated by sum_k path_k mu_layer[k][e]. */
void or_brem_spectrum_layered(int64_t n_seg, const double *E_keV, const double *L_ang,
                              const double *r_mid, const double *v_hat, int n_el, const double *Z,
                              const double *n_ang3, const or_layer_escape *layers, const double n_hat[3],
                              int64_t n_e, const double *E_grid, const double *mu_layer, double *spec,
                              int n_threads);

/* Escape pieces of one segment (segment_escape.py:193-272 with layers):
 * returns the piece count P (<= 8) and writes frac[P], path0[P*K], path1[P*K]. */
int or_layer_pieces(double z0, double z1, const or_layer_escape *ly, double n_z, double *frac,
                    double *path0, double *path1);

#ifdef __cplusplus
}
#endif
#endif
