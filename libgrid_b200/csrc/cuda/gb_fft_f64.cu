// FP64 instantiation of the line-pass FFT schedules.
#include <string.h>

#include "gb_fft_drv.cuh"

template int gb__fft3d_t<double>(void *, const gb_geom *, int, double);
template int gb__split_step_t<double>(void *, const gb_geom *, const gb_kinetic *, const gb_potential *);
template int gb__split_steps_t<double>(void *, const gb_geom *, const gb_kinetic *, const gb_potential *, int);
template int gb__ksq_sum_t<double>(const void *, void *, const gb_geom *, double *);
