// mpmw_internal.cuh -- host-side launchers shared between the library's
// translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include "../../include/mpmw.h"
#include "../../include/mpmw_xpbd.h"

namespace mpmw {

int launch_stress(const mpmw_particles_t &p, const mpmw_params_t &prm, cudaStream_t s);
int launch_p2g(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st, cudaStream_t s);
int launch_g2p(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st, bool fused,
               void *ws, size_t ws_bytes, cudaStream_t s);
// chained: launched as the fused schedule's programmatic dependent launches,
// with the worklist count already reset by the grid pass before it
int launch_g2p2g(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st,
                 bool store_stress, void *ws, size_t ws_bytes, cudaStream_t s, bool chained = false);
size_t g2p_workspace_bytes(int64_t n);
int launch_stress_p2g(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st,
                      void *ws, size_t ws_bytes, cudaStream_t s);
size_t hash_workspace_bytes(int64_t n);
size_t block_sort_workspace_bytes(int64_t n);
int block_sort(const float *x, int64_t n, const mpmw_params_t &prm, const int32_t *dims, int block, int32_t *perm,
               void *ws, size_t ws_bytes, cudaStream_t s);
int reserve_fused_smem();
size_t batch_workspace_bytes(const mpmw_grid_t *grids, int nscenes, int64_t n);
int prepare_batch(const mpmw_particles_t &p, const mpmw_grid_t *grids, const mpmw_params_t *prms,
                  const int64_t *offsets, int nscenes, void *ws, size_t ws_bytes, cudaStream_t s);
bool set_batch_options(const void *ws, int gather_tile, int read_ahead);
int launch_batch_substeps(const mpmw_particles_t &p, int first, int last, int nsteps, uint32_t *st, void *ws,
                          size_t ws_bytes, cudaStream_t s);
// the fused substeps of all scenes in one persistent (cooperative) launch
int launch_batch_persistent(const mpmw_particles_t &p, int nsteps, uint32_t *st, void *ws, size_t ws_bytes,
                            cudaStream_t s);
int64_t batch_persistent_launches();

}  // namespace mpmw
