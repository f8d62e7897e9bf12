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

// Record the message pb_last_error() returns on this thread.
void set_last_error(const char *msg);

}  // namespace pb
