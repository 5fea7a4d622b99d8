/*
 * argot_b200_legacy.h -- the older GPU entry-point names of ARGOT for the
 * point-source path, exported by libargot_b200_legacy.so, a thin shim over
 * libargot_b200.so.
 *
 * ARGOT's src/step_radiation.c (:162,172,326,336,492) calls the GPU march
 * and rate functions of src/calc_optical_depth.cu:30 and
 * src/calc_photoion_rate.cu:95 under the same names as their CPU versions
 * (src/prototype.h:66-67).  A GPU build of that driver links this library
 * in place of those two objects; a CPU build must not link it (the names
 * would collide).  Semantics, errors and threading are those of
 * calc_optical_depth_cuda / calc_photoion_rate_cuda in argot_b200.h.
 */
#ifndef ARGOT_B200_LEGACY_H
#define ARGOT_B200_LEGACY_H

#include "argot_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces src/calc_optical_depth.cu:29-144 (the same contract as
 * calc_optical_depth_cuda). */
ARGOT_B200_API void calc_optical_depth(struct ray_segment *seg, struct cuda_mem_space *cuda_mem,
                                       struct cuda_param *this_cuda, struct run_param *this_run);

/* Replaces src/calc_photoion_rate.cu:94-216 (the same contract as
 * calc_photoion_rate_cuda). */
ARGOT_B200_API void calc_photoion_rate(struct cuda_mem_space *cuda_mem, struct light_ray *ray,
                                       struct light_ray_IO *ray_IO, struct cuda_param *this_cuda,
                                       struct run_param *this_run);

#ifdef __cplusplus
}
#endif

#endif /* ARGOT_B200_LEGACY_H */
