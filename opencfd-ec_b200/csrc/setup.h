// Host-side interface of the setup kernels (setup.cu).
#pragma once
#include <cuda_runtime.h>

#include "arena.h"

namespace ocfd {

struct GeoArgs {
  const BlkD* blk;
  int nblk;
  const long long *pre_face, *pre_cell, *pre_box;
  long long tot_face, tot_cell, tot_box, tot_node;
  const double *x, *y, *z;  // node coordinates with the ghost layer filled
  double* M;                // M_COUNT planes of tot_face
  double* scratch;          // >= 3*tot_face doubles
  double *vol, *dtm, *dw;   // cell
  double *xc, *yc, *zc;     // box
  const double* Xw;         // wall nodes (3 per node) or null, grouped by solve
  long long nwall;
  const long long* wpre;    // nsolve + 1: wall nodes of solve q are [wpre[q], wpre[q+1])
  const struct WallChunk* wch;  // chunks of consecutive wall nodes with their bounding boxes
  const int* wcpre;         // nsolve + 1: chunks of solve q are [wcpre[q], wcpre[q+1])
};

// a run of up to 64 consecutive wall nodes of one solve and its axis-aligned bounding box
struct WallChunk {
  double lo[3], hi[3];
  long long w0, w1;
};

cudaError_t run_geometry(const GeoArgs& a, cudaStream_t st);
cudaError_t convert_to_float(const double* src, float* dst, long long n, cudaStream_t st);

}  // namespace ocfd
