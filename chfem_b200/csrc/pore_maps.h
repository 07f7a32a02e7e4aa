// pore_maps.h -- host entry of the device Stokes DOF-number maps (pore_maps.cu).
#pragma once
#include <cstdint>
#include <algorithm>
#include <cuda_runtime.h>

namespace chfem {

struct PoreColorMap { int16_t mat[256]; };  // material index of each colour, -1 when unlisted

// Fluid keys (d_fk, N bytes) from the colours, and the chunk counts of pore and interface nodes
// scanned in place (d_cnt, 2 x pore_maps_chunks(N)); returns the counts nV and nB.
bool pore_maps_count(const uint8_t* d_colors, const PoreColorMap& cm, int R, int C, int L, int ref, uint8_t* d_fk,
                     unsigned* d_cnt, unsigned long long* d_tot, int* d_bad, unsigned long long* nV, unsigned long long* nB,
                     cudaStream_t st, const char** err);
// The maps from the keys and the scanned counts: dof_of_node (N), node_of_dof (nV + nB),
// border keys (nB).
bool pore_maps_number(const uint8_t* d_fk, int R, int C, int L, const unsigned* d_cnt, unsigned nV, uint32_t* d_dof_of_node,
                      uint32_t* d_node_of_dof, uint8_t* d_border, cudaStream_t st, const char** err);
long pore_maps_chunks(long N);

}  // namespace chfem
