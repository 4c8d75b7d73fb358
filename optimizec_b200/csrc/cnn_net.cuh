// cnn_net.cuh — the hidden and last layers of the closure network in one persistent launch.
//
// Layers 1 .. L-1 of the tensor-core network (cnn_tc.cuh) run as one cooperative kernel with one
// CTA per SM.  Work items are (layer, image, tile row, 128-pixel strip) tiles, numbered layer by
// layer; CTA c takes tiles c, c + G, c + 2G, ... (G CTAs) in that order.  A tile of layer l >= 2
// needs the tile rows t - 1, t, t + 1 (periodic) of layer l - 1 in every strip; each finished
// tile counts once in a per-(layer, image, tile row) counter, and the producer waits (bounded)
// for the three counters before it loads the halo.  Every dependency of a tile has a smaller
// number, every CTA takes its tiles in increasing order and every CTA is resident, so the
// smallest unfinished tile can always proceed and the waits end.  The same waits
// also cover the reuse of the two activation buffers: layer l writes the buffer layer l - 2
// wrote, and every tile of layer l - 1 that reads those rows (its own dependencies) has finished
// before layer l's tile starts.
//
// Inside a CTA the roles are warp-specialised and pipelined:
//   producer warp: dependency wait (one poll checks the three input-row counters of the next
//     kNetLookahead tiles, three lanes each, with acquire loads), then one thread issues one bulk
//     copy (cp.async.bulk) of the tile's contiguous halo run into one of `stages` halo buffers,
//     completing on that stage's mbarrier;
//   MMA issuer (one thread): 24 tcgen05.mma per tile (issue_conv_tile) into one of 4 TMEM
//     accumulator buffers, committed to the stage's "empty" barrier and the buffer's "full"
//     barrier;
//   16 epilogue warps in two groups of 8 taking alternate tiles: in a group, warp w reads TMEM
//     lanes 32 (w % 4) .. + 31 (pixels) x 32 columns (channels) of tile row (w / 4) % 2, frees
//     the buffer, adds the bias, applies GELU and stores the bf16 pixel (with its halo copies);
//     the group then meets at its named barrier and one thread releases the tile (red.release),
//     or for the last layer the warps write the f32 output times the output scale; while one
//     group's releasing thread waits for the stores, the rest go on.
// Layer l takes its tile rows in the order l - 1, l, ..., so that every tile's input rows come at
// most two rows after its own position in the previous layer (no wait on the previous layer's
// last rows at the periodic wrap).
// So the halo copies of tile i + 1, the MMAs of tile i and the epilogue of tile i - 1 overlap,
// and no kernel boundary separates the layers.  The weights of all layers stay in shared memory.
// Every wait is bounded: a wait that runs out sets *err, the producer then hands out an end
// marker, every role stops, the copies and MMAs in flight are waited for (bounded) and the tensor
// memory is freed.  The last CTA to finish resets the counters for the next launch.
#pragma once
#include "cnn_tc.cuh"

namespace dns2d {
namespace cnntc {

constexpr int kNetMaxLayers = 8;                      // network depth the launch supports
constexpr int kNetEpiWarps = 16;                      // epilogue warps: two groups taking alternate tiles
constexpr int kNetGroupWarps = 8;                     // warps of a group (two per TMEM lane quadrant)
constexpr int kNetThreads = (kNetEpiWarps + 2) * 32;  // + producer warp + MMA warp
constexpr int kNetMaxStages = 4;                      // halo buffers
constexpr int kNetBufs = 4;                           // TMEM accumulator buffers of TR x 32 columns
constexpr int kNetTmemCols = kNetBufs * TR * C;       // 256
// a halo stage holds one tile's contiguous halo run ([row][plane][pixel], A_BYTES); stages start
// on 1024-byte boundaries
constexpr int kNetHaloTx = A_BYTES;                   // 33 280 bytes one stage's copy delivers
constexpr int kNetStage = (kNetHaloTx + 1023) / 1024 * 1024;
constexpr int kNetWHidden = TcShape<32>::B_BYTES;     // 18 432
constexpr int kNetWLast = TcShape<16>::B_BYTES;       // 9 216
constexpr long long kNetSpinLimit = 1ll << 22;        // polls of a dependency counter
constexpr int kNetTraceSlots = 10;                    // timestamps per tile of a traced launch
constexpr int kNetLookahead = 10;                     // tiles whose input rows one poll checks

__host__ __device__ constexpr size_t net_weight_bytes(int L) { return (size_t)(L - 2) * kNetWHidden + kNetWLast; }
__host__ __device__ constexpr size_t net_stage_offset(int L) { return (net_weight_bytes(L) + 1023) / 1024 * 1024; }
// dynamic shared memory of the launch: 1 KB of slack to align the base, weights, stages
__host__ __device__ constexpr size_t net_smem_bytes(int L, int stages)
{
    return 1024 + net_stage_offset(L) + (size_t)stages * kNetStage;
}

struct NetLaunch {
    const __nv_bfloat16 *wtc = nullptr;  // layers 1 .. L-2 [dx][chunk][2 - dy][32][8], then layer L-1 with 16
    const float *bias[kNetMaxLayers] = {};  // bias of layer l (l = 1 .. L-1)
    __nv_bfloat16 *act[2] = {nullptr, nullptr};  // strip layout; layer 0 wrote act[0], layer l < L-1 writes act[l & 1]
    float *yf = nullptr;                 // last layer: [B][H][W] f32
    float out_scale = 1.0f;
    int L = 0, B = 0, H = 0, W = 0;
    int stages = 2;
    unsigned int *sync = nullptr;        // [0] CTAs finished, [1 ..] (L-2) x B x (H / TR) row counters
    int *err = nullptr;                  // set to 1 when a wait runs out
    long long spin_limit = kNetSpinLimit;
    unsigned long long *trace = nullptr;  // optional: kNetTraceSlots timestamps per tile (cnn_net.cu, trace_at)
};

// counters of one launch: finished CTAs and one per (layer 1 .. L-2, image, tile row)
__host__ __device__ inline size_t net_sync_words(int L, int B, int H) { return 1 + (size_t)(L - 2) * B * (H / TR); }

// host side (cnn_net.cu): cooperative launch of one CTA per SM; returns the CUDA error
cudaError_t net_launch(const NetLaunch &q, cudaStream_t stream, int *grid_out);
// shared-memory stages that fit for a depth-L network (0: the network does not fit)
int net_stages_that_fit(int L);

}  // namespace cnntc
}  // namespace dns2d
