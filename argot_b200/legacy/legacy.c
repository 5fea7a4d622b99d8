/* legacy.c -- libargot_b200_legacy.so: ARGOT's older GPU entry-point names
 * (src/calc_optical_depth.cu:30, src/calc_photoion_rate.cu:95) forwarded to
 * libargot_b200.so (include/argot_b200_legacy.h). */
#include "argot_b200_legacy.h"

void calc_optical_depth(struct ray_segment *seg, struct cuda_mem_space *cuda_mem, struct cuda_param *this_cuda,
                        struct run_param *this_run) {
  calc_optical_depth_cuda(seg, cuda_mem, this_cuda, this_run);
}

void calc_photoion_rate(struct cuda_mem_space *cuda_mem, struct light_ray *ray, struct light_ray_IO *ray_IO,
                        struct cuda_param *this_cuda, struct run_param *this_run) {
  calc_photoion_rate_cuda(cuda_mem, ray, ray_IO, this_cuda, this_run);
}
