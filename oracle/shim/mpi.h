/*
 * Single-rank stand-in for the subset of MPI that ARGOT's ray-tracing hot
 * path calls (test infrastructure only: it lets the reference's own
 * calc_optical_depth.c / accum_optical_depth.c / assign_ray_segment.c /
 * calc_photoion_rate.c / smooth_photoion_rate.c and the diffuse-radiation
 * sources of src/diffuse_photon be compiled and run on one host without an
 * MPI library).
 *
 * Semantics with one rank (rank 0 of a world of size 1):
 *  - MPI_Win_create records the window base and displacement unit, so that
 *    MPI_Put / MPI_Accumulate to rank 0 act on local memory exactly as a real
 *    MPI would (assign_ray_segment.c relies on a Put to itself to learn its
 *    own segment count).
 *  - MPI_Allgather / MPI_Gather / MPI_Bcast copy or do nothing.
 *  - Fences and barriers are no-ops.
 */
#ifndef ARGOT_ORACLE_MPI_SHIM_H
#define ARGOT_ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef ptrdiff_t MPI_Aint;
typedef struct { int dummy; } *MPI_Info;
typedef struct argot_shim_win { char *base; size_t size; int disp_unit; } *MPI_Win;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_BYTE 1
#define MPI_FLOAT 2
#define MPI_UINT64_T 3
#define MPI_INT 4
#define MPI_DOUBLE 5
#define MPI_SUM 1
#define MPI_MODE_NOPRECEDE 1
#define MPI_MODE_NOSUCCEED 2
#define MPI_MODE_NOSTORE 4

/* a derived datatype of n bytes (the reference builds its struct types with
 * MPI_Type_struct; here the driver sets them to their byte size) */
#define ARGOT_SHIM_SIZED_TYPE(n) (0x10000 + (int)(n))

static inline size_t argot_shim_type_size(MPI_Datatype t)
{
  if (t >= 0x10000) return (size_t)(t - 0x10000);
  switch (t) {
  case MPI_BYTE: return 1;
  case MPI_FLOAT: return 4;
  case MPI_UINT64_T: return 8;
  case MPI_INT: return 4;
  case MPI_DOUBLE: return 8;
  default: return 1;
  }
}

static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }

static inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r,
                                int rc, MPI_Datatype rt, MPI_Comm c)
{
  (void)rc; (void)rt; (void)c;
  memmove(r, s, (size_t)sc * argot_shim_type_size(st));
  return MPI_SUCCESS;
}

static inline int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r,
                             int rc, MPI_Datatype rt, int root, MPI_Comm c)
{
  (void)rc; (void)rt; (void)root; (void)c;
  memmove(r, s, (size_t)sc * argot_shim_type_size(st));
  return MPI_SUCCESS;
}

static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
  (void)b; (void)n; (void)t; (void)root; (void)c;
  return MPI_SUCCESS;
}

static struct { int dummy; } argot_shim_info_obj;

static inline int MPI_Info_create(MPI_Info *i) { *i = (MPI_Info)&argot_shim_info_obj; return MPI_SUCCESS; }
static inline int MPI_Info_set(MPI_Info i, const char *k, const char *v) { (void)i; (void)k; (void)v; return MPI_SUCCESS; }
static inline int MPI_Info_free(MPI_Info *i) { *i = NULL; return MPI_SUCCESS; }

#include <stdlib.h>
static inline int MPI_Win_create(void *base, MPI_Aint size, int disp_unit,
                                 MPI_Info info, MPI_Comm c, MPI_Win *w)
{
  (void)info; (void)c;
  *w = (MPI_Win)malloc(sizeof(struct argot_shim_win));
  (*w)->base = (char *)base;
  (*w)->size = (size_t)size;
  (*w)->disp_unit = disp_unit;
  return MPI_SUCCESS;
}

static inline int MPI_Win_fence(int assert_, MPI_Win w) { (void)assert_; (void)w; return MPI_SUCCESS; }
static inline int MPI_Win_free(MPI_Win *w) { free(*w); *w = NULL; return MPI_SUCCESS; }

static inline int MPI_Put(const void *o, int oc, MPI_Datatype ot, int rank,
                          MPI_Aint disp, int tc, MPI_Datatype tt, MPI_Win w)
{
  (void)rank; (void)tc; (void)tt;
  memmove(w->base + (size_t)disp * (size_t)w->disp_unit, o,
          (size_t)oc * argot_shim_type_size(ot));
  return MPI_SUCCESS;
}

static inline int MPI_Accumulate(const void *o, int oc, MPI_Datatype ot, int rank,
                                 MPI_Aint disp, int tc, MPI_Datatype tt, MPI_Op op,
                                 MPI_Win w)
{
  (void)rank; (void)tc; (void)tt; (void)op;
  if (ot == MPI_FLOAT) {
    float *dst = (float *)(w->base + (size_t)disp * (size_t)w->disp_unit);
    const float *src = (const float *)o;
    for (int i = 0; i < oc; i++) dst[i] += src[i];
  }
  return MPI_SUCCESS;
}

/* memory for windows, and the struct datatype of the diffuse-radiation
 * code (src/diffuse_photon/diffuse_photon_mpi.c): one block of `count`
 * elements of one basic type, sized here */
static inline int MPI_Alloc_mem(MPI_Aint size, MPI_Info info, void *baseptr)
{
  (void)info;
  *(void **)baseptr = malloc((size_t)size);
  return MPI_SUCCESS;
}
static inline int MPI_Free_mem(void *base) { free(base); return MPI_SUCCESS; }
static inline int MPI_Type_struct(int n, const int *blocklen, const MPI_Aint *disp,
                                  const MPI_Datatype *types, MPI_Datatype *out)
{
  size_t bytes = 0;
  for (int i = 0; i < n; i++)
    bytes = (size_t)disp[i] + (size_t)blocklen[i] * argot_shim_type_size(types[i]);
  *out = ARGOT_SHIM_SIZED_TYPE(bytes);
  return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }

#endif /* ARGOT_ORACLE_MPI_SHIM_H */
