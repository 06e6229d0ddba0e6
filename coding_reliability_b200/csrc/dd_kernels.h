// dd_kernels.h — host-side declarations of the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "dd_jobs.h"

namespace dd {

// How a lane bumps its shared-memory bin: one fire-and-forget shared atomic
// (red.shared.add) or a load/add/store on its private column.
enum HistMode : int { HIST_RED = 0, HIST_LDST = 1 };

size_t hist_smem_bytes(uint32_t smem_bins, bool col_table);
cudaError_t hist_occupancy(int mode, size_t smem, int* ctas_per_sm);
cudaError_t launch_hist(int mode, const LaunchArgs& args, int grid, size_t smem, cudaStream_t stream);
cudaError_t launch_popc_rate(uint32_t iters, int grid, uint32_t* sink, cudaStream_t stream);
// pattern 0: per-thread columns (the single tcgen05 epilogue); 1: lane columns shared by all warps (the paired one)
cudaError_t launch_red_rate(uint32_t iters, int grid, int threads, int pattern, uint32_t* sink, cudaStream_t stream);
uint64_t red_rate_adds(uint32_t iters, int grid, int threads);
cudaError_t launch_plain(uint64_t A, uint64_t N, uint32_t nbins, unsigned long long* bins, int grid,
                         cudaStream_t stream);

}  // namespace dd
