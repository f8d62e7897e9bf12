// Internal launch interfaces shared by the pyrite_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/pyrite_b200.h"

namespace pb {

// Largest LUT staged into shared memory by the transport kernel.
constexpr size_t kLutSmemBytes = 192 * 1024;

cudaError_t launch_transport(const pb_transport_args &a, cudaStream_t s, int sms);
cudaError_t launch_cxr(const pb_cxr_args &a, cudaStream_t s, int sms);
cudaError_t launch_brem(const pb_brem_args &a, cudaStream_t s, int sms);
cudaError_t launch_char(const pb_char_args &a, cudaStream_t s, int sms);
cudaError_t launch_char_spectrum(int n_dir, int n_line, int n_E, const double *yield, const double *profiles,
                                 double *spec, cudaStream_t s);

cudaError_t launch_mlp_gemm(const pb_mlp_gemm_args &g, cudaStream_t s);
cudaError_t launch_mlp_mse_grad(int rows, int cols, const float *Y, const void *T, int64_t ldt_in, float t_scale,
                                float g_scale, void *dY, void *dYt, int64_t ld_t, float *loss, cudaStream_t s);
cudaError_t launch_mlp_colsum(int rows, int cols, const float *X, int64_t ld, float *out, cudaStream_t s);
cudaError_t launch_mlp_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                            float eps, float wd, float bc1, float bc2, cudaStream_t s);
cudaError_t launch_mlp_pack(int rows, int cols, const float *W, void *Wb, int ldb, void *Wt, int ldt, int pad_cols,
                            cudaStream_t s);

cudaError_t launch_mlp_infer(const pb_mlp_infer_args &a, cudaStream_t s, int sms);
cudaError_t launch_mlp_head(int n_dir, int n_out, const float *W5, const float *b5, const double *hsum,
                            const double *lsum, double t_scale, double *spec, cudaStream_t s);
cudaError_t launch_mlp_pack_umma(int cols, int kc, const float *W, void *out, cudaStream_t s);

cudaError_t launch_bin_lines(int64_t n_lines, const double *line_E, const double *line_a, const double *line_w,
                             const int32_t *line_dir, const int64_t *line_seg, int dir0, int n_dir_chunk,
                             int64_t n_seg, double lo, double width, int n_bins, float *target, cudaStream_t st);
cudaError_t launch_mlp_features(const pb_mlp_infer_args &a, void *X, float *weight, cudaStream_t s);

cudaError_t launch_mlp_group_mse_grad(int groups, int S, int cols, const float *Y, const void *T, int64_t ldt_in,
                                      const float *w, float t_scale, float g_scale, void *dY, void *dYt, int64_t ld_t,
                                      float *loss, cudaStream_t s);

cudaError_t launch_segments_sample(const pb_segments &src, int64_t stride, const pb_segments &dst,
                                   unsigned int *status, cudaStream_t s, int sms);

uint64_t coherent_work_bytes(int n_row, int64_t n_line, int n_E);
// Work items (x-blocks of the field kernel) of a coherent reduction.
int64_t coherent_items(int n_row, int64_t n_line, int n_E);
cudaError_t launch_coherent(const pb_coherent_args &a, cudaStream_t s);
uint64_t coherent_blend_work_bytes(int n_row, int64_t n_line, int n_E);
cudaError_t launch_coherent_blend(const pb_coherent_blend_args &a, cudaStream_t s);
cudaError_t launch_decoherence(const pb_decoherence_args &a, cudaStream_t s);
cudaError_t launch_coherent_accumulate(const pb_coherent_stream_args &a, cudaStream_t s);
cudaError_t launch_coherent_stream_finalize(int n_row, int n_E, const double *w_row, const double *fields,
                                            const double *power, const double *F_row, double scale, double *spec,
                                            cudaStream_t s);

uint64_t coherent_records_work_bytes(int64_t n_seg, int n_g);
cudaError_t launch_coherent_records(const pb_coherent_records_args &r, cudaStream_t s, int sms);

// Record the message pb_last_error() returns on this thread.
void set_last_error(const char *msg);

// Host checks of a pb_cxr_args, shared by every scorer entry point: PB_OK, or
// an error code with pb_last_error() set ("who: ..."). own_far_workspace: the
// entry point supplies the far-field workspace itself.
int validate_cxr(const pb_cxr_args &a, const char *who, bool own_far_workspace);

}  // namespace pb
