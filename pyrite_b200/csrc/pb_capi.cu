// C ABI of pyrite_b200: argument checks, error reporting, launches.
//
// Every entry point validates its plain-C arguments on the host, launches on
// the caller's stream and returns a pb_status. Errors carry a message in a
// thread-local buffer read by pb_last_error(). Nothing here allocates.
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "pb_brem_node.cuh"
#include "pb_internal.h"

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    return fail(PB_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

// Streaming multiprocessors of the current device (cached per device).
int device_sms() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

}  // namespace

namespace pb {
void set_last_error(const char *msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }

int validate_cxr(const pb_cxr_args &a, const char *who, bool own_far_workspace) {
    if (a.n_seg < 0 || a.n_dir < 1 || a.n_E < 1)
        return fail(PB_ERR_INVALID, "%s: need n_seg >= 0, n_dir >= 1, n_E >= 1", who);
    if (a.n_seg == 0) return PB_OK;
    if (a.precision != PB_FP64 && a.precision != PB_MIXED)
        return fail(PB_ERR_INVALID, "%s: unknown precision %d", who, a.precision);
    const pb_cxr_tables &t = a.tables;
    if (t.n_g < 1 || t.n_tab < 2 || t.n_mu < 1 || t.n_mu > 4)
        return fail(PB_ERR_INVALID, "%s: need n_g >= 1, n_tab >= 2, 1 <= n_mu <= 4", who);
    if (!t.G || !t.ES || !t.EP || !t.WM || !t.row_table || !t.E_tab || !t.chi_re || !t.chi_im ||
        !t.u_re || !t.u_im || !t.log_mu || !t.delta)
        return fail(PB_ERR_INVALID, "%s: every table pointer must be set", who);
    if (!a.n_hat || !a.r_mid || !a.v_hat || !a.L || !a.E_keV || !a.elec_id)
        return fail(PB_ERR_INVALID, "%s: segment and direction pointers must be set", who);
    if (a.quadrature == PB_QUAD_BINMEAN) {
        if (!a.edges || !a.spec) return fail(PB_ERR_INVALID, "%s: bin-mean needs edges and spec", who);
        if (a.exact_widths > 0.0 && a.far_pad >= 0 && !a.far_moments && !own_far_workspace)
            return fail(PB_ERR_INVALID, "%s: far field needs the far_moments workspace", who);
    } else if (a.quadrature == PB_QUAD_NODE) {
        if (!a.line_E || !a.line_a || !a.line_w || !a.line_dir || !a.line_count)
            return fail(PB_ERR_INVALID, "%s: node quadrature needs a line buffer", who);
        if (a.spec && !a.E_grid) return fail(PB_ERR_INVALID, "%s: node spectrum needs E_grid", who);
    } else {
        return fail(PB_ERR_INVALID, "%s: unknown quadrature %d", who, a.quadrature);
    }
    // A line buffer (bin-mean or node) is written through line_count: all of
    // its arrays and a positive capacity, or none.
    if (a.line_E && (!a.line_count || a.line_capacity < 1 || !a.line_a || !a.line_w || !a.line_dir))
        return fail(PB_ERR_INVALID, "%s: line buffer needs line_E/a/w/dir, a count and a capacity >= 1", who);
    if (a.n_layer < 0 || a.n_layer > 4)
        return fail(PB_ERR_UNSUPPORTED, "%s: n_layer = %d outside [0, 4]", who, a.n_layer);
    if (a.n_layer > 0 && (!a.z_top || !a.z_bot || !a.mu_off || !a.mu_knot || !a.mu_value || !a.mu_slope))
        return fail(PB_ERR_INVALID, "%s: a layered absorber needs bounds and mu tables", who);
    return PB_OK;
}
}  // namespace pb

extern "C" {

int pb_abi_version(void) { return PB_ABI_VERSION; }

const char *pb_last_error(void) { return g_err; }

int pb_device_count(int *count) {
    if (!count) return fail(PB_ERR_INVALID, "pb_device_count: count is NULL");
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    return PB_OK;
}

// Argument checks of pb_transport (no CUDA call); n == 0 passes.
static int check_transport(const pb_transport_args *a) {
    if (!a) return fail(PB_ERR_INVALID, "pb_transport: args is NULL");
    if (a->n < 0) return fail(PB_ERR_INVALID, "pb_transport: n = %lld < 0", (long long)a->n);
    if (a->n == 0) return PB_OK;
    if (a->layers.n_layers < 1 || a->layers.n_layers > 8)
        return fail(PB_ERR_INVALID, "pb_transport: n_layers = %d outside [1, 8]", a->layers.n_layers);
    if (a->layers.max_el < 1 || a->layers.max_el > 8)
        return fail(PB_ERR_INVALID, "pb_transport: max_el = %d outside [1, 8]", a->layers.max_el);
    if (!a->layers.z_top || !a->layers.z_bot || !a->layers.n_el || !a->layers.J || !a->layers.k ||
        !a->layers.coeff || !a->layers.E_cross || !a->layers.sr_rate_numer || !a->layers.sr_joy_numer)
        return fail(PB_ERR_INVALID, "pb_transport: layer tables must all be set");
    if (!a->work_counter) return fail(PB_ERR_INVALID, "pb_transport: work_counter is NULL");
    if (a->rng != PB_RNG_SPLITMIX && a->rng != PB_RNG_PHILOX)
        return fail(PB_ERR_INVALID, "pb_transport: unknown rng %d", a->rng);
    if (a->precision != PB_FP64 && a->precision != PB_MIXED)
        return fail(PB_ERR_INVALID, "pb_transport: unknown precision %d", a->precision);
    if (a->use_lut) {
        const int eb = a->precision == PB_MIXED ? 4 : 8;
        if (!a->lut.base || a->lut.elem_bytes != eb)
            return fail(PB_ERR_INVALID, "pb_transport: LUT needs %d-byte values for this precision", eb);
        if (a->lut.n_energy < 2) return fail(PB_ERR_INVALID, "pb_transport: LUT n_energy < 2");
        if (a->lut.total_bytes % 16 != 0 || ((uintptr_t)a->lut.base % 16) != 0)
            return fail(PB_ERR_INVALID, "pb_transport: LUT buffer must be 16-byte aligned and sized");
    }
    if (a->beam.mode == PB_BEAM_EXPLICIT && (!a->beam.pos0 || !a->beam.dir0 || !a->beam.E0))
        return fail(PB_ERR_INVALID, "pb_transport: explicit beam needs pos0, dir0 and E0");
    if (a->beam.mode < 0 || a->beam.mode > 2)
        return fail(PB_ERR_INVALID, "pb_transport: unknown beam mode %d", a->beam.mode);
    if (a->rows.L && a->cap < 1) return fail(PB_ERR_INVALID, "pb_transport: rows need cap >= 1");
    if (a->seg.L && (!a->seg.count || a->seg.capacity < 0))
        return fail(PB_ERR_INVALID, "pb_transport: segment list needs a count and a capacity");
    if (a->tallies.exit_E && (a->tallies.n_E < 1 || a->tallies.n_E > 256))
        return fail(PB_ERR_INVALID, "pb_transport: exit energy bins must be in [1, 256]");
    if (a->tallies.exit_theta && (a->tallies.n_theta < 1 || a->tallies.n_theta > 256))
        return fail(PB_ERR_INVALID, "pb_transport: exit angle bins must be in [1, 256]");
    if (a->block_threads != 0 && (a->block_threads % 32 != 0 || a->block_threads > 256))
        return fail(PB_ERR_INVALID, "pb_transport: block_threads must be a multiple of 32 <= 256");
    if (a->straggling && !a->Z) return fail(PB_ERR_INVALID, "pb_transport: straggling needs Z");
    if (a->elastic_model != PB_ELASTIC_SR && a->elastic_model != PB_ELASTIC_ELSEPA)
        return fail(PB_ERR_INVALID, "pb_transport: elastic_model = %d", a->elastic_model);
    if (a->elastic_model == PB_ELASTIC_ELSEPA) {
        const pb_elsepa &t = a->elsepa;
        if (a->use_lut) return fail(PB_ERR_UNSUPPORTED, "pb_transport: ELSEPA elastic runs on the exact core only");
        if (t.n_mu < 2 || t.cells < 1 || (t.cells & (t.cells - 1)))
            return fail(PB_ERR_INVALID, "pb_transport: ELSEPA needs n_mu >= 2 and a power-of-two cell count");
        if (!t.start || !t.length || !t.logE || !t.log_rate || !t.cdf || !t.pdf || !t.mu || !t.guide)
            return fail(PB_ERR_INVALID, "pb_transport: every ELSEPA table pointer must be set");
    }
    if (a->stopping.count) {
        if (a->use_lut) return fail(PB_ERR_UNSUPPORTED, "pb_transport: SBETHE stopping runs on the exact core only");
        if (a->stopping.width < 2 || !a->stopping.logE || !a->stopping.logS)
            return fail(PB_ERR_INVALID, "pb_transport: SBETHE tables need width >= 2, logE and logS");
    }
    return PB_OK;
}

static int run_transport(const pb_transport_args *a, cudaStream_t s) {
    if (a->n == 0) return PB_OK;
    cudaError_t e = cudaMemsetAsync(a->work_counter, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(e, "pb_transport: zero work counter");
    e = pb::launch_transport(*a, s, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_transport: launch");
    return PB_OK;
}

int pb_transport(const pb_transport_args *a, void *stream) {
    const int v = check_transport(a);
    return v != PB_OK ? v : run_transport(a, (cudaStream_t)stream);
}

int pb_cxr_score(const pb_cxr_args *a, void *stream) {
    if (!a) return fail(PB_ERR_INVALID, "pb_cxr_score: args is NULL");
    const int v = pb::validate_cxr(*a, "pb_cxr_score", false);
    if (v != PB_OK || a->n_seg == 0) return v;
    cudaError_t e = pb::launch_cxr(*a, (cudaStream_t)stream, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_cxr_score: launch");
    return PB_OK;
}

static int check_brem(const pb_brem_args *a) {
    if (!a) return fail(PB_ERR_INVALID, "pb_brem_score: args is NULL");
    if (a->n_seg < 0 || a->n_dir < 1 || a->n_E < 1)
        return fail(PB_ERR_INVALID, "pb_brem_score: need n_seg >= 0, n_dir >= 1, n_E >= 1");
    if (a->n_seg == 0) return PB_OK;
    if (a->n_el < 1 || a->n_el > 4) return fail(PB_ERR_INVALID, "pb_brem_score: 1 <= n_el <= 4");
    if (a->n_layer < 0 || a->n_layer > 4)
        return fail(PB_ERR_UNSUPPORTED, "pb_brem_score: n_layer = %d outside [0, 4]", a->n_layer);
    if (a->n_layer > 0 && (!a->z_top || !a->z_bot || !a->mu_layer))
        return fail(PB_ERR_INVALID, "pb_brem_score: a layered absorber needs bounds and mu_layer");
    if (!a->n_hat || !a->r_mid || !a->v_hat || !a->L || !a->E_keV || !a->elec_id || !a->Z ||
        !a->n_ang3 || !a->E_grid || (!a->mu && a->n_layer == 0) || !a->spec)
        return fail(PB_ERR_INVALID, "pb_brem_score: every pointer must be set");
    if (a->work != nullptr && pb::brem_node_applies(*a)) {
        const int64_t need = (int64_t)pb::brem_node_layout(*a).total;
        if (a->work_bytes < need)
            return fail(PB_ERR_INVALID, "pb_brem_score: work_bytes %lld below the %lld pb_brem_work_size gives",
                        (long long)a->work_bytes, (long long)need);
        if (((uintptr_t)a->work & 15u) != 0) return fail(PB_ERR_INVALID, "pb_brem_score: work is not 16-byte aligned");
    }
    return PB_OK;
}

int pb_brem_work_size(const pb_brem_args *a, int64_t *bytes) {
    if (!a || !bytes) return fail(PB_ERR_INVALID, "pb_brem_work_size: args or bytes is NULL");
    if (a->n_seg < 0 || a->n_E < 1 || a->n_el < 1 || a->n_el > 4)
        return fail(PB_ERR_INVALID, "pb_brem_work_size: need n_seg >= 0, n_E >= 1, 1 <= n_el <= 4");
    *bytes = pb::brem_node_applies(*a) ? (int64_t)pb::brem_node_layout(*a).total : 0;
    return PB_OK;
}

static int run_brem(const pb_brem_args *a, cudaStream_t s) {
    if (a->n_seg == 0) return PB_OK;
    cudaError_t e = pb::launch_brem(*a, s, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_brem_score: launch");
    return PB_OK;
}

int pb_brem_score(const pb_brem_args *a, void *stream) {
    const int v = check_brem(a);
    return v != PB_OK ? v : run_brem(a, (cudaStream_t)stream);
}

static int check_char(const pb_char_args *a) {
    if (!a) return fail(PB_ERR_INVALID, "pb_char_yields: args is NULL");
    if (a->n_seg < 0 || a->n_dir < 1 || a->n_line < 1 || a->n_shell < 1)
        return fail(PB_ERR_INVALID, "pb_char_yields: need n_seg >= 0, n_dir >= 1, n_line >= 1, n_shell >= 1");
    if (a->n_seg == 0) return PB_OK;
    if (a->n_shell > 40 || a->n_line > 256 || a->n_layer < 0 || a->n_layer > 8)
        return fail(PB_ERR_UNSUPPORTED, "pb_char_yields: n_shell <= 40, n_line <= 256, 0 <= n_layer <= 8");
    if ((size_t)a->n_dir * (size_t)a->n_line * sizeof(double) > 200 * 1024)
        return fail(PB_ERR_UNSUPPORTED, "pb_char_yields: n_dir * n_line above the shared accumulator");
    if (a->precision != PB_FP64 && a->precision != PB_MIXED)
        return fail(PB_ERR_INVALID, "pb_char_yields: unknown precision");
    if (!a->n_hat || !a->r_mid || !a->v_hat || !a->L || !a->E_keV || !a->elec_id || !a->shell_E ||
        !a->shell_sigma || !a->shell_offset || !a->response || !a->mu || !a->line_yield)
        return fail(PB_ERR_INVALID, "pb_char_yields: every table, segment and output pointer must be set");
    if (a->n_layer > 0 && (!a->z_top || !a->z_bot))
        return fail(PB_ERR_INVALID, "pb_char_yields: layer bounds missing");
    if (a->n_layer == 0 && !(a->thickness > 0.0))
        return fail(PB_ERR_INVALID, "pb_char_yields: single slab needs thickness > 0");
    return PB_OK;
}

static int run_char(const pb_char_args *a, cudaStream_t s) {
    if (a->n_seg == 0) return PB_OK;
    cudaError_t e = pb::launch_char(*a, s, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_char_yields: launch");
    return PB_OK;
}

int pb_char_yields(const pb_char_args *a, void *stream) {
    const int v = check_char(a);
    return v != PB_OK ? v : run_char(a, (cudaStream_t)stream);
}

int pb_transport_score(const pb_transport_score_args *p, void *stream) {
    if (!p) return fail(PB_ERR_INVALID, "pb_transport_score: args is NULL");
    if (p->n_cxr < 0 || p->n_brem < 0 || p->n_char < 0 || (p->n_cxr && !p->cxr) || (p->n_brem && !p->brem) ||
        (p->n_char && !p->chars))
        return fail(PB_ERR_INVALID, "pb_transport_score: scorer counts and arrays disagree");
    if (!p->transport.seg.L || !p->transport.seg.count)
        return fail(PB_ERR_INVALID, "pb_transport_score: the transport needs its segment stream");
    // every check before any launch
    int v = check_transport(&p->transport);
    for (int i = 0; v == PB_OK && i < p->n_cxr; ++i) v = pb::validate_cxr(p->cxr[i], "pb_transport_score (cxr)", false);
    for (int i = 0; v == PB_OK && i < p->n_brem; ++i) v = check_brem(&p->brem[i]);
    for (int i = 0; v == PB_OK && i < p->n_char; ++i) v = check_char(&p->chars[i]);
    if (v != PB_OK) return v;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(p->transport.seg.count, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(e, "pb_transport_score: zero the segment count");
    if ((v = run_transport(&p->transport, s)) != PB_OK) return v;
    for (int i = 0; i < p->n_cxr; ++i) {
        if (p->cxr[i].n_seg == 0) continue;
        e = pb::launch_cxr(p->cxr[i], s, device_sms());
        if (e != cudaSuccess) return cuda_fail(e, "pb_transport_score: cxr launch");
    }
    for (int i = 0; i < p->n_brem; ++i)
        if ((v = run_brem(&p->brem[i], s)) != PB_OK) return v;
    for (int i = 0; i < p->n_char; ++i)
        if ((v = run_char(&p->chars[i], s)) != PB_OK) return v;
    return PB_OK;
}

int pb_char_spectrum(int32_t n_dir, int32_t n_line, int32_t n_E, const double *line_yield, const double *profiles,
                     double *spec, void *stream) {
    if (n_dir < 1 || n_line < 1 || n_E < 1 || n_dir > 65535)
        return fail(PB_ERR_INVALID, "pb_char_spectrum: need 1 <= n_dir <= 65535, n_line >= 1, n_E >= 1");
    if (!line_yield || !profiles || !spec) return fail(PB_ERR_INVALID, "pb_char_spectrum: pointers must be set");
    cudaError_t e = pb::launch_char_spectrum(n_dir, n_line, n_E, line_yield, profiles, spec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_char_spectrum: launch");
    return PB_OK;
}

int pb_mlp_gemm(const pb_mlp_gemm_args *g, void *stream) {
    if (!g) return fail(PB_ERR_INVALID, "pb_mlp_gemm: args is NULL");
    if (g->M < 1 || g->N < 1 || g->K < 16 || g->K % 16 != 0)
        return fail(PB_ERR_INVALID, "pb_mlp_gemm: need M, N >= 1 and K a positive multiple of 16");
    if (!g->A || !g->B) return fail(PB_ERR_INVALID, "pb_mlp_gemm: A and B must be set");
    if (g->lda < g->K || g->ldb < g->K || g->lda % 8 != 0 || g->ldb % 8 != 0 ||
        ((uintptr_t)g->A & 15u) != 0 || ((uintptr_t)g->B & 15u) != 0)
        return fail(PB_ERR_INVALID, "pb_mlp_gemm: lda, ldb >= K, multiples of 8, operands 16-byte aligned");
    if ((g->out_f32 && g->ldc < g->N) || (g->out_bf16 && g->ldh < g->N) || (g->out_bf16_t && g->ldt < g->M) ||
        (g->dsilu_z && g->ldz < g->N))
        return fail(PB_ERR_INVALID, "pb_mlp_gemm: an output leading dimension is too small");
    if (g->act != 0 && g->act != 1) return fail(PB_ERR_INVALID, "pb_mlp_gemm: act is 0 or 1");
    cudaError_t e = pb::launch_mlp_gemm(*g, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_gemm: launch");
    return PB_OK;
}

int pb_mlp_mse_grad(int32_t rows, int32_t cols, const float *Y, const void *T, int64_t ldt_in, float t_scale,
                    float g_scale, void *dY, void *dYt, int64_t ld_t, float *loss, void *stream) {
    if (rows < 1 || cols < 1 || !Y || !T || !dY || !dYt || !loss || ldt_in < cols || ld_t < rows)
        return fail(PB_ERR_INVALID, "pb_mlp_mse_grad: bad sizes or pointers");
    cudaError_t e = pb::launch_mlp_mse_grad(rows, cols, Y, T, ldt_in, t_scale, g_scale, dY, dYt, ld_t, loss,
                                            (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_mse_grad: launch");
    return PB_OK;
}

int pb_mlp_group_mse_grad(int32_t groups, int32_t S, int32_t cols, const float *Y, const void *T, int64_t ldt_in,
                          const float *w, float t_scale, float g_scale, void *dY, void *dYt, int64_t ld_t,
                          float *loss, void *stream) {
    if (groups < 1 || groups > 65535 || S < 1 || cols < 1 || !Y || !T || !w || !dY || !dYt || !loss ||
        ldt_in < cols || ld_t < (int64_t)groups * S)
        return fail(PB_ERR_INVALID, "pb_mlp_group_mse_grad: bad sizes or pointers");
    cudaError_t e = pb::launch_mlp_group_mse_grad(groups, S, cols, Y, T, ldt_in, w, t_scale, g_scale, dY, dYt, ld_t,
                                                  loss, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_group_mse_grad: launch");
    return PB_OK;
}

int pb_mlp_colsum(int32_t rows, int32_t cols, const float *X, int64_t ld, float *out, void *stream) {
    if (rows < 1 || cols < 1 || !X || !out || ld < cols) return fail(PB_ERR_INVALID, "pb_mlp_colsum: bad arguments");
    cudaError_t e = pb::launch_mlp_colsum(rows, cols, X, ld, out, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_colsum: launch");
    return PB_OK;
}

int pb_mlp_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                float wd, float bc1, float bc2, void *stream) {
    if (n < 1 || !p || !g || !m || !v) return fail(PB_ERR_INVALID, "pb_mlp_adam: bad arguments");
    cudaError_t e = pb::launch_mlp_adam(n, p, g, m, v, lr, b1, b2, eps, wd, bc1, bc2, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_adam: launch");
    return PB_OK;
}

int pb_mlp_pack(int32_t rows, int32_t cols, const float *W, void *Wb, int32_t ldb, void *Wt, int32_t ldt,
                int32_t pad_cols, void *stream) {
    if (rows < 1 || cols < 1 || !W || !Wb || ldb < cols || (Wt && (ldt < rows || pad_cols < 1 || pad_cols > ldb)))
        return fail(PB_ERR_INVALID, "pb_mlp_pack: bad arguments");
    cudaError_t e = pb::launch_mlp_pack(rows, cols, W, Wb, ldb, Wt, ldt, pad_cols, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_pack: launch");
    return PB_OK;
}

int pb_segments_sample(const pb_segments *src, int64_t stride, const pb_segments *dst, unsigned int *status,
                       void *stream) {
    if (!src || !dst || stride < 1) return fail(PB_ERR_INVALID, "pb_segments_sample: need src, dst, stride >= 1");
    if (!src->count || !src->r_mid || !src->v_hat || !src->L || !src->E_repr || !src->elec_id || !dst->count ||
        !dst->r_mid || !dst->v_hat || !dst->L || !dst->E_repr || !dst->elec_id || src->capacity < 0 ||
        dst->capacity < 0)
        return fail(PB_ERR_INVALID, "pb_segments_sample: segment arrays must be set");
    cudaError_t e = pb::launch_segments_sample(*src, stride, *dst, status, (cudaStream_t)stream, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_segments_sample: launch");
    return PB_OK;
}

namespace {
// One block per range (grid-strided): 16-byte moves where both ends and the
// length allow, bytes otherwise.
__global__ void __launch_bounds__(256) copy_segments_kernel(int n, const int64_t *desc) {
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const unsigned char *src = reinterpret_cast<const unsigned char *>(desc[3 * k]);
        unsigned char *dst = reinterpret_cast<unsigned char *>(desc[3 * k + 1]);
        const int64_t nb = desc[3 * k + 2];
        int64_t done = 0;
        if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0) {
            const int64_t n16 = nb >> 4;
            for (int64_t i = threadIdx.x; i < n16; i += blockDim.x)
                reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
            done = n16 << 4;
        }
        for (int64_t i = done + threadIdx.x; i < nb; i += blockDim.x) dst[i] = src[i];
    }
}
}  // namespace

int pb_copy_segments(int32_t n, const int64_t *desc, void *stream) {
    if (n < 0 || (n > 0 && !desc)) return fail(PB_ERR_INVALID, "pb_copy_segments: need n >= 0 and desc");
    if (n == 0) return PB_OK;
    const int grid = n < 4 * device_sms() ? n : 4 * device_sms();
    copy_segments_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(n, desc);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pb_copy_segments: launch");
    return PB_OK;
}

int pb_mlp_infer(const pb_mlp_infer_args *a, void *stream) {
    if (!a) return fail(PB_ERR_INVALID, "pb_mlp_infer: args is NULL");
    if (a->n_seg < 0 || a->n_dir < 1) return fail(PB_ERR_INVALID, "pb_mlp_infer: need n_seg >= 0, n_dir >= 1");
    if (a->n_seg == 0) return PB_OK;
    if (!a->dir_uv || !a->r_mid || !a->v_hat || !a->L || !a->E_keV || !a->elec_id || !a->w1_packed ||
        !a->w_packed[0] || !a->w_packed[1] || !a->w_packed[2] || !a->bias[0] || !a->bias[1] || !a->bias[2] ||
        !a->bias[3] || !a->hsum || !a->lsum)
        return fail(PB_ERR_INVALID, "pb_mlp_infer: every pointer must be set");
    if (((uintptr_t)a->w1_packed & 15u) || ((uintptr_t)a->w_packed[0] & 15u) || ((uintptr_t)a->w_packed[1] & 15u) ||
        ((uintptr_t)a->w_packed[2] & 15u))
        return fail(PB_ERR_INVALID, "pb_mlp_infer: packed weights must be 16-byte aligned");
    if (!(a->theta_max > 0.0) || !(a->E_hi_MeV > a->E_lo_MeV) || !(a->E_lo_MeV > 0.0) || !(a->thickness > 0.0))
        return fail(PB_ERR_INVALID, "pb_mlp_infer: need theta_max > 0, 0 < E_lo < E_hi, thickness > 0");
    cudaError_t e = pb::launch_mlp_infer(*a, (cudaStream_t)stream, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_infer: launch");
    return PB_OK;
}

int pb_mlp_head(int32_t n_dir, int32_t n_out, const float *W5, const float *b5, const double *hsum,
                const double *lsum, double t_scale, double *spec, void *stream) {
    if (n_dir < 1 || n_dir > 65535 || n_out < 1 || !W5 || !b5 || !hsum || !lsum || !spec)
        return fail(PB_ERR_INVALID, "pb_mlp_head: bad arguments");
    cudaError_t e = pb::launch_mlp_head(n_dir, n_out, W5, b5, hsum, lsum, t_scale, spec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_head: launch");
    return PB_OK;
}

int pb_mlp_pack_umma(int32_t cols, int32_t kc, const float *W, void *out, void *stream) {
    if (cols < 1 || (kc != 16 && kc != 32 && kc != 64) || !W || !out)
        return fail(PB_ERR_INVALID, "pb_mlp_pack_umma: bad arguments");
    cudaError_t e = pb::launch_mlp_pack_umma(cols, kc, W, out, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_pack_umma: launch");
    return PB_OK;
}

int pb_mlp_features(const pb_mlp_infer_args *a, void *X, float *weight, void *stream) {
    if (!a || !X || a->n_seg < 1 || a->n_dir < 1 || !a->dir_uv || !a->r_mid || !a->v_hat || !a->L || !a->E_keV ||
        !a->elec_id || !(a->theta_max > 0.0) || !(a->E_hi_MeV > a->E_lo_MeV) || !(a->E_lo_MeV > 0.0) ||
        !(a->thickness > 0.0))
        return fail(PB_ERR_INVALID, "pb_mlp_features: bad arguments");
    cudaError_t e = pb::launch_mlp_features(*a, X, weight, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_mlp_features: launch");
    return PB_OK;
}

int pb_cxr_bin_lines(int64_t n_lines, const double *line_E, const double *line_a, const double *line_w,
                     const int32_t *line_dir, const int64_t *line_seg, int32_t dir0, int32_t n_dir_chunk,
                     int64_t n_seg, double lo_eV, double width_eV, int32_t n_bins, float *target, void *stream) {
    if (n_lines < 0 || n_dir_chunk < 1 || n_seg < 1 || n_bins < 1 || !(width_eV > 0.0))
        return fail(PB_ERR_INVALID, "pb_cxr_bin_lines: bad sizes");
    if (n_lines > 0 && (!line_E || !line_a || !line_w || !line_dir || !line_seg || !target))
        return fail(PB_ERR_INVALID, "pb_cxr_bin_lines: pointers must be set");
    cudaError_t e = pb::launch_bin_lines(n_lines, line_E, line_a, line_w, line_dir, line_seg, dir0, n_dir_chunk,
                                         n_seg, lo_eV, width_eV, n_bins, target, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_cxr_bin_lines: launch");
    return PB_OK;
}

// Sizes the coherent reduction accepts: one energy-tile grid dimension, an
// int item count, the items kernel's 1024-thread row split.
static int coherent_sizes_ok(int32_t n_row, int64_t n_line, int32_t n_E) {
    return n_row >= 1 && n_row <= (1 << 24) && n_line >= 0 && n_line <= (int64_t(1) << 40) && n_E >= 1 &&
           n_E <= (1 << 24);
}

// The field kernel's grid has one x-block per work item: at most 2^31 - 1.
// Every size coherent_sizes_ok accepts stays far below it (items <= n_row +
// 148 * 3 * 4); the check guards the launch should those limits change.
static int coherent_grid_ok(int32_t n_row, int64_t n_line, int32_t n_E) {
    return pb::coherent_items(n_row, n_line, n_E) <= (int64_t)INT32_MAX;
}

int pb_coherent_records_work_size(int64_t n_seg, int32_t n_g, uint64_t *bytes) {
    if (!bytes) return fail(PB_ERR_INVALID, "pb_coherent_records_work_size: bytes is NULL");
    if (n_seg < 0 || n_g < 1 || (n_g > 0 && n_seg > (int64_t)INT32_MAX))
        return fail(PB_ERR_INVALID, "pb_coherent_records_work_size: need 0 <= n_seg < 2^31, n_g >= 1");
    *bytes = pb::coherent_records_work_bytes(n_seg, n_g);
    return PB_OK;
}

int pb_coherent_records(const pb_coherent_records_args *r, void *stream) {
    if (!r) return fail(PB_ERR_INVALID, "pb_coherent_records: args is NULL");
    const pb_cxr_args &a = r->cxr;
    if (a.n_dir != 1) return fail(PB_ERR_INVALID, "pb_coherent_records: one direction per call (n_dir = 1)");
    if (a.n_seg < 0 || a.n_seg > (int64_t)INT32_MAX)
        return fail(PB_ERR_INVALID, "pb_coherent_records: need 0 <= n_seg < 2^31");
    const pb_cxr_tables &t = a.tables;
    if (t.n_g < 1 || t.n_tab < 2 || t.n_mu < 1 || t.n_mu > 4 || !t.G || !t.ES || !t.EP || !t.WM ||
        !t.row_table || !t.E_tab || !t.chi_re || !t.chi_im || !t.u_re || !t.u_im || !t.log_mu || !t.delta)
        return fail(PB_ERR_INVALID, "pb_coherent_records: incomplete reflection tables");
    if (a.n_layer != 0) return fail(PB_ERR_UNSUPPORTED, "pb_coherent_records: single slab only (n_layer = 0)");
    if (!r->row_off) return fail(PB_ERR_INVALID, "pb_coherent_records: row_off must be set");
    if (a.n_seg == 0) {
        cudaError_t e = cudaMemsetAsync(r->row_off, 0, sizeof(int64_t) * ((size_t)t.n_g + 1), (cudaStream_t)stream);
        return e == cudaSuccess ? PB_OK : cuda_fail(e, "pb_coherent_records: zero row_off");
    }
    if (!a.n_hat || !a.r_mid || !a.v_hat || !a.L || !a.E_keV || !a.elec_id)
        return fail(PB_ERR_INVALID, "pb_coherent_records: segment and direction pointers must be set");
    if (r->capacity < 0 || (r->capacity > 0 && (!r->E_vac || !r->a_vac || !r->phase_slope || !r->g_phase ||
                                                 !r->cs_re || !r->cs_im || !r->cp_re || !r->cp_im || !r->L_esc ||
                                                 !r->half_dL || !r->apb || !r->bma || !r->q)))
        return fail(PB_ERR_INVALID, "pb_coherent_records: every record array must be set for capacity > 0");
    if (!r->work || reinterpret_cast<uintptr_t>(r->work) % 256 != 0)
        return fail(PB_ERR_INVALID, "pb_coherent_records: work must be set and 256-byte aligned");
    const uint64_t need = pb::coherent_records_work_bytes(a.n_seg, t.n_g);
    if (r->work_bytes < need)
        return fail(PB_ERR_CAPACITY, "pb_coherent_records: work holds %llu bytes, needs %llu",
                    (unsigned long long)r->work_bytes, (unsigned long long)need);
    cudaError_t e = pb::launch_coherent_records(*r, (cudaStream_t)stream, device_sms());
    if (e != cudaSuccess) return cuda_fail(e, "pb_coherent_records: launch");
    return PB_OK;
}

int pb_coherent_work_size(int32_t n_row, int64_t n_line, int32_t n_E, uint64_t *bytes) {
    if (!bytes) return fail(PB_ERR_INVALID, "pb_coherent_work_size: bytes is NULL");
    if (!coherent_sizes_ok(n_row, n_line, n_E))
        return fail(PB_ERR_INVALID, "pb_coherent_work_size: need 1 <= n_row, n_E <= 2^24 and 0 <= n_line <= 2^40");
    if (!coherent_grid_ok(n_row, n_line, n_E))
        return fail(PB_ERR_UNSUPPORTED, "pb_coherent_work_size: more than 2^31 - 1 work items; split the rows");
    *bytes = pb::coherent_work_bytes(n_row, n_line, n_E);
    return PB_OK;
}

static int coherent_check(const pb_coherent_args *a, const char *who, uint64_t need) {
    if (!coherent_sizes_ok(a->n_row, a->n_line, a->n_E))
        return fail(PB_ERR_INVALID, "%s: need 1 <= n_row, n_E <= 2^24 and 0 <= n_line <= 2^40", who);
    if (!coherent_grid_ok(a->n_row, a->n_line, a->n_E))
        return fail(PB_ERR_UNSUPPORTED, "%s: more than 2^31 - 1 work items; split the rows", who);
    if (!a->row_off || !a->row_weight || !a->E || !a->delta_omega || !a->spec || !a->work)
        return fail(PB_ERR_INVALID, "%s: row_off, row_weight, E, delta_omega, spec, work must be set", who);
    if (a->n_line > 0 && (!a->E_vac || !a->a_vac || !a->phase_slope || !a->g_phase || !a->cs_re || !a->cs_im ||
                          !a->cp_re || !a->cp_im || !a->L_esc || !a->half_dL || !a->apb || !a->bma || !a->q))
        return fail(PB_ERR_INVALID, "%s: every line record array must be set", who);
    if (reinterpret_cast<uintptr_t>(a->work) % 256 != 0)
        return fail(PB_ERR_INVALID, "%s: work must be 256-byte aligned", who);
    if (!(a->sinc_cutoff >= 0.0)) return fail(PB_ERR_INVALID, "%s: sinc_cutoff must be >= 0", who);
    if (a->work_bytes < need)
        return fail(PB_ERR_CAPACITY, "%s: work holds %llu bytes, needs %llu", who,
                    (unsigned long long)a->work_bytes, (unsigned long long)need);
    return PB_OK;
}

int pb_coherent_blend_work_size(int32_t n_row, int64_t n_line, int32_t n_E, uint64_t *bytes) {
    if (!bytes) return fail(PB_ERR_INVALID, "pb_coherent_blend_work_size: bytes is NULL");
    if (!coherent_sizes_ok(n_row, n_line, n_E))
        return fail(PB_ERR_INVALID,
                    "pb_coherent_blend_work_size: need 1 <= n_row, n_E <= 2^24 and 0 <= n_line <= 2^40");
    if (!coherent_grid_ok(n_row, n_line, n_E))
        return fail(PB_ERR_UNSUPPORTED, "pb_coherent_blend_work_size: more than 2^31 - 1 work items; split the rows");
    *bytes = pb::coherent_blend_work_bytes(n_row, n_line, n_E);
    return PB_OK;
}

int pb_coherent_blend(const pb_coherent_blend_args *b, void *stream) {
    if (!b) return fail(PB_ERR_INVALID, "pb_coherent_blend: args is NULL");
    const pb_coherent_args *a = &b->base;
    if (!coherent_sizes_ok(a->n_row, a->n_line, a->n_E))
        return fail(PB_ERR_INVALID, "pb_coherent_blend: need 1 <= n_row, n_E <= 2^24 and 0 <= n_line <= 2^40");
    const int rc = coherent_check(a, "pb_coherent_blend", pb::coherent_blend_work_bytes(a->n_row, a->n_line, a->n_E));
    if (rc != PB_OK) return rc;
    if (!b->F_row || (a->n_line > 0 && !b->elec_id))
        return fail(PB_ERR_INVALID, "pb_coherent_blend: elec_id and F_row must be set");
    if (a->n_line == 0) return PB_OK;
    cudaError_t e = pb::launch_coherent_blend(*b, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_coherent_blend: launch");
    return PB_OK;
}

int pb_coherent_accumulate(const pb_coherent_stream_args *b, void *stream) {
    if (!b) return fail(PB_ERR_INVALID, "pb_coherent_accumulate: args is NULL");
    const pb_coherent_args *a = &b->base;
    if (!coherent_sizes_ok(a->n_row, a->n_line, a->n_E))
        return fail(PB_ERR_INVALID, "pb_coherent_accumulate: need 1 <= n_row, n_E <= 2^24 and 0 <= n_line <= 2^40");
    const uint64_t need = b->elec_id ? pb::coherent_blend_work_bytes(a->n_row, a->n_line, a->n_E)
                                     : pb::coherent_work_bytes(a->n_row, a->n_line, a->n_E);
    pb_coherent_args chk = *a;
    double dummy_spec = 0.0;
    if (!chk.spec) chk.spec = &dummy_spec;  // the accumulation writes no spectrum
    const int rc = coherent_check(&chk, "pb_coherent_accumulate", need);
    if (rc != PB_OK) return rc;
    if (!b->fields || (b->elec_id && !b->power))
        return fail(PB_ERR_INVALID, "pb_coherent_accumulate: fields (and power with elec_id) must be set");
    if (a->n_line == 0) return PB_OK;
    cudaError_t e = pb::launch_coherent_accumulate(*b, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_coherent_accumulate: launch");
    return PB_OK;
}

int pb_coherent_finalize(int32_t n_row, int32_t n_E, const double *row_weight, const double *fields,
                         const double *power, const double *F_row, double scale, double *spec, void *stream) {
    if (n_row < 1 || n_E < 1 || n_E > (1 << 24) || !row_weight || !fields || !spec || (F_row && !power))
        return fail(PB_ERR_INVALID, "pb_coherent_finalize: need n_row, n_E >= 1, row_weight, fields, spec "
                                    "(and power with F_row)");
    cudaError_t e = pb::launch_coherent_stream_finalize(n_row, n_E, row_weight, fields, power, F_row, scale, spec,
                                                        (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_coherent_finalize: launch");
    return PB_OK;
}

int pb_decoherence_factor(const pb_decoherence_args *a, void *stream) {
    if (!a) return fail(PB_ERR_INVALID, "pb_decoherence_factor: args is NULL");
    if (a->n_row < 1 || a->n_row > 65535 || a->n_pop < 1 || a->n_E < 1 || a->n_E > (1 << 24))
        return fail(PB_ERR_INVALID, "pb_decoherence_factor: need 1 <= n_row <= 65535, n_pop >= 1, 1 <= n_E <= 2^24");
    if (!a->G || !a->A_pop || !a->xy0_pop || !a->omega || !a->F)
        return fail(PB_ERR_INVALID, "pb_decoherence_factor: G, A_pop, xy0_pop, omega and F must be set");
    cudaError_t e = pb::launch_decoherence(*a, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_decoherence_factor: launch");
    return PB_OK;
}

int pb_coherent_reduce(const pb_coherent_args *a, void *stream) {
    if (!a) return fail(PB_ERR_INVALID, "pb_coherent_reduce: args is NULL");
    if (!coherent_sizes_ok(a->n_row, a->n_line, a->n_E))
        return fail(PB_ERR_INVALID, "pb_coherent_reduce: need 1 <= n_row, n_E <= 2^24 and 0 <= n_line <= 2^40");
    const int rc = coherent_check(a, "pb_coherent_reduce", pb::coherent_work_bytes(a->n_row, a->n_line, a->n_E));
    if (rc != PB_OK) return rc;
    if (a->n_line == 0) return PB_OK;  // no line: the spectrum is unchanged
    cudaError_t e = pb::launch_coherent(*a, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "pb_coherent_reduce: launch");
    return PB_OK;
}

}  // extern "C"
