// FP32 instantiation of the line-pass FFT schedules (FP32 mode: FP32 storage,
// FFT and elementwise arithmetic; phase arguments reduced in FP64).
#include <string.h>

#include "gb_fft_drv.cuh"

template int gb__fft3d_t<float>(void *, const gb_geom *, int, double);
template int gb__split_step_t<float>(void *, const gb_geom *, const gb_kinetic *, const gb_potential *);
template int gb__split_steps_t<float>(void *, const gb_geom *, const gb_kinetic *, const gb_potential *, int);
template int gb__ksq_sum_t<float>(const void *, void *, const gb_geom *, double *);
