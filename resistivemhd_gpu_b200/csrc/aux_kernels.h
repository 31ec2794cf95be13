// aux_kernels.h -- launchers for the boundary fill, CFL reduction and layout
// conversion kernels of librmhd2d (aux_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "rmhd2d_internal.h"

namespace rmhd2d {

void launch_boundary(const Grid &g, double *s, const double *row2, Control *ctl, int slot, cudaStream_t st);
void launch_boundary_batch(const BatchRun *runs, int nruns, long long max_ghost, int which, int slot, cudaStream_t st);
void launch_snapshot_row2(const Grid &g, const double *s, double *row2, cudaStream_t st);
void launch_rate(const Grid &g, const double *s, Control *ctl, int slot, int set_crash, cudaStream_t st);
// Slabs of a decomposed domain: halo columns to / from a packed buffer, the
// domain's ghost column 0 held in the first slab's halo, the control words
// combined across slabs.
void launch_slab_halo(const Grid &g, double *s, double *buf, int col0, int to_buf, cudaStream_t st);
void launch_slab_origin_column(const Grid &g, double *s, Control *ctl, int slot, cudaStream_t st);
void launch_slab_words(Control *ctl, int slot, long long *w, int to_buf, cudaStream_t st);
void launch_aos_to_planes(const Grid &g, const double *aos, double *s, cudaStream_t st);
void launch_planes_to_aos(const Grid &g, const double *s, double *aos, cudaStream_t st);
void launch_table_to_plane(const Grid &g, const double *tab, double *plane, cudaStream_t st);

}  // namespace rmhd2d
