// Tiled AO kernels (ao_tile.cu): tables and launchers.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "kernels.cuh"

namespace qb {

constexpr int kTilePoints = 32;   // points per CTA
constexpr int kTileShells = 32;   // shells per AO tile (at most)
constexpr int kTileNuc = 32;      // nuclei per AO tile (at most)

// AO tiles: consecutive AO ranges starting on multiples of 8, 64 AOs wide (32
// where 64 AOs would span more than 32 shells or nuclei).  Built when AOs are
// numbered shell by shell and shells nucleus by nucleus (ntiles = 0 otherwise).
struct AoTiles {
  int32_t ntiles = 0;
  const int4* tile = nullptr;       // (k_begin, k_end, shell_begin, shell_end)
  const int2* tile_nuc = nullptr;   // (nuc_begin, nuc_end)
  const int32_t* ao_tcode = nullptr;  // a | b<<4 | c<<8 | l<<12 | shell_local<<16 | nuc_local<<21
};

cudaError_t launch_ao_tile_f64(const DevTables& T, const AoTiles& Tl, int64_t P, const double* coord, double cutoff,
                               bool dp_exp, int comps, double* out, cudaStream_t s);
// AO pieces (split.cuh) of rows (point, component); scales: the scale block
// of the coefficient pieces (its AO-component scales are used).
cudaError_t launch_ao_tile_split(const DevTables& T, const AoTiles& Tl, int64_t P, const double* coord, double cutoff,
                                 int comps, int pieces, const double* scales, void* a, int64_t lda,
                                 int64_t piece_stride, cudaStream_t s);

}  // namespace qb
