// dd_mma.h — the tcgen05 (5th-gen tensor core) path: AN exhaustive, grid and Ext-Hamming all-pairs jobs.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "dd_jobs.h"

namespace dd {

struct MmaArgs {
  const Job* jobs;
  uint32_t njobs;
  uint32_t hist_rows;        // bin rows in shared memory: >= every job's nbins and operand bits + 1
  uint64_t total_tiles;      // work items: (super tile, 128-row strip) as in the popc kernel
  unsigned long long* counter;
  unsigned* status;          // KSTATUS_* bits, zeroed before the launch
  unsigned long long timeout_ns;  // bound of every mbarrier wait
  uint32_t b_bufs;           // column-operand buffers in shared memory: 2 when they fit next to the bins, else 1
  uint32_t packed;           // 1: pair-packed epilogue (two distances per MMA column, joint-bin table)
  uint32_t pk_cells;         // pair-packed: joint-table cells of this launch (S x window rows of its jobs)
  uint32_t pad;
};

// True if the job can run on the MMA path: all pairs of a codeword progression or
// of the Ext-Hamming codewords, or a grid of lattice rows and progression / lattice
// columns; at most 60 operand bits.
bool mma_eligible(const Job& j);
// Operand bit planes L of job j; its distances lie in [0, L].
int mma_operand_bits(const Job& j);
// Largest distance of job j's pairs: the bit count of its widest codeword.
int mma_max_distance(const Job& j);
// Pair-packed launch layout for jobs whose largest S is smax: a joint table of
// every (d1, d2) cell (smax^2) beside two column-operand buffers when that fits
// in shared memory, else as many cells as fit beside one buffer.
void mma_pk_layout(uint32_t smax, uint32_t* cells, uint32_t* b_bufs);
// Pair-packed epilogue parameters of job j in a table of `cells` cells:
// pk_s = largest distance + 1; the window of d2 - pk_lo in [0, W), W = the whole
// rows of S cells that fit, centred on the mean distance of a fixed sample of
// the job's pairs; pk_limit = S * W.  The window only affects speed: values
// outside it are counted as two single distances.
void mma_pack_setup(Job& j, uint32_t cells);
// Column-operand buffers that fit in shared memory next to the bins (single epilogue).
uint32_t mma_b_bufs(uint32_t hist_rows);
size_t mma_smem_bytes(uint32_t hist_rows, uint32_t b_bufs, bool packed, uint32_t pk_cells);
cudaError_t launch_mma(const MmaArgs& args, int grid, size_t smem, cudaStream_t stream);

}  // namespace dd
