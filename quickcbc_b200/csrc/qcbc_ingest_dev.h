// Device-side pieces of the input stage shared with qcbc_capi.cu: the PSD model's makespec into
// device rows, and the rebuild of an event's weighted data after its PSD changed.
#pragma once
#include <cuda_runtime.h>

#include "../../include/qcbc_ingest.h"

namespace qcbc {

int psd_model_nifo(const qcbc_psd_model* m);
// makespec of sample k for every detector into d_S rows (stride doubles apart), queued on s.
int psd_model_draw_dev(qcbc_psd_model* m, int k, double Tobs, int N, double* d_S, int stride, cudaStream_t s);

// Smallest positive PSD of each detector over bins [lo, hi) (HUGE_VAL when none), into d_out[nifo].
void launch_band_min(const double* d_S, int stride, int nifo, int lo, int hi, double* d_out, cudaStream_t s);

struct Sigmas {
  double v[3];
};
// Weighted data of bins [lo, hi) from D [nifo][N] and S rows: 4 sigma D/S (real, imaginary),
// 4 sigma^2 / S, in FP64 ([nifo][3][nh]) and, times the bin factors i^{-7/6}, i^{-7/6}, i^{-7/3},
// in the mixed kernel's FP32 planes (EventData::wm).  Bins outside [lo, hi) are left as they are.
void launch_event_weights(const double* d_D, int N, const double* d_S, int stride, int nifo, int lo, int hi,
                          Sigmas sigma, double* d_w64, float* d_wm, cudaStream_t s);

}  // namespace qcbc
