// cnn_net.cu — the persistent, warp-specialised network launch (cnn_net.cuh): device roles and
// the cooperative host launch.
#include "cnn_net.cuh"

#include <algorithm>

namespace dns2d {
namespace cnntc {
namespace {

struct Item {
    int l, b, t, xs;
};

__device__ __forceinline__ Item decode(int item, int B, int T, int S)
{
    const int per_layer = B * T * S;
    Item it;
    const int j = item / per_layer;
    int r = item - j * per_layer;
    it.l = j + 1;
    it.b = r / (T * S);
    r -= it.b * (T * S);
    const int pos = r / S;
    it.xs = r - pos * S;
    it.t = (pos + j) % T;  // layer l starts at tile row l - 1
    return it;
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Wait until tile `item` (and as many of the next kNetLookahead - 1 tiles of this CTA, every G
// tiles, as are ready too) has its input rows complete: lanes 3j, 3j + 1, 3j + 2 read the
// counters of tile rows t - 1, t, t + 1 of layer l - 1 for the tile j steps ahead (acquire loads;
// every strip releases into them).  Returns how many consecutive tiles from `item` are ready
// (>= 1), or 0 when the wait ran out or another wait did (recorded in *err).
__device__ int net_deps(const NetLaunch &q, int item, int G, int total, int T, int S, unsigned int need, int lane)
{
    const int j = lane / 3, d = lane - 3 * (lane / 3);
    const unsigned int *c = nullptr;
    const int it_j = item + j * G;
    if (j < kNetLookahead && it_j < total) {
        const Item it = decode(it_j, q.B, T, S);
        if (it.l >= 2) c = q.sync + 1 + ((size_t)(it.l - 2) * q.B + it.b) * T + (it.t + d - 1 + T) % T;
    }
    long long n = 0;
    for (;;) {
        const bool ok = c == nullptr || ld_acquire_u32(c) >= need;
        const unsigned int mask = __ballot_sync(0xffffffffu, ok);
        int m = 0;
        while (m < kNetLookahead && ((mask >> (3 * m)) & 7u) == 7u) ++m;
        if (m > 0) {
            __syncwarp();  // the lanes' acquires are ordered before lane 0's copies
            return m;
        }
        const int e = __shfl_sync(0xffffffffu, lane == 0 ? *(volatile int *)q.err : 0, 0);
        if (e != 0) return 0;
        if (++n > q.spin_limit) {
            if (lane == 0) atomicExch(q.err, 1);
            return 0;
        }
        __nanosleep(64);
    }
}

// optional per-tile timestamps (globaltimer ns): producer [0] took the tile, [1] its input
// rows complete, [2] its stage free, [3] copy issued; MMA issuer [4] copy landed, [5] MMAs
// issued and committed (after the accumulator buffer was free); warp 0 of the tile's epilogue
// group [6] started, [7] read the accumulator, [8] issued its stores, [9] released the tile (or
// wrote its output)
__device__ __forceinline__ void trace_at(const NetLaunch &q, int item, int j)
{
    if (q.trace) q.trace[(size_t)item * kNetTraceSlots + j] = global_ns();
}

// AND of p over an epilogue group's 256 threads at its named barrier 1 + grp: the group takes
// every decision together, so no warp of it can be left waiting at the group's barrier
__device__ __forceinline__ bool group_all(bool p, int grp)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(1 + grp), "r"(kNetGroupWarps * 32)
        : "memory");
    return r != 0;
}

// An epilogue group's release of a finished tile: every warp orders its stores for the async
// proxy, the group meets at its named barrier (1 + grp, the group's 256 threads), and one thread
// releases the tile-row counter (cumulative over the group's stores seen through the barrier).
// The other warps go on to their next tile without waiting for the stores.
__device__ __forceinline__ void net_release(const NetLaunch &q, int idx, int grp, bool leader)
{
    fence_proxy_async_global();
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(kNetGroupWarps * 32) : "memory");
    if (leader) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(q.sync + idx) : "memory");
}

__global__ void __launch_bounds__(kNetThreads, 1) k_cnn_net(const __grid_constant__ NetLaunch q)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t full[kNetMaxStages], empty[kNetMaxStages], tfull[kNetBufs], tempty[kNetBufs], wbar;
    __shared__ int info[kNetMaxStages], tinfo[kNetBufs];
    __shared__ uint32_t tmem_holder;
    __shared__ int s_last;
    __shared__ float sbias[kNetMaxLayers][C];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int L = q.L, NS = q.stages;
    const int T = q.H / TR, S = q.W / TM;
    const int total = (L - 1) * q.B * T * S;
    unsigned char *base = sm + ((1024u - (saddr(sm) & 1023u)) & 1023u);  // 1024-byte aligned
    unsigned char *sW = base;                          // weights of layers 1 .. L-1
    unsigned char *sStage = base + net_stage_offset(L);  // NS halo stages of kNetStage bytes

    for (int e = tid; e < (L - 1) * C; e += kNetThreads) {
        const int l = 1 + e / C, co = e % C;
        sbias[l][co] = (l < L - 1 || co == 0) ? q.bias[l][co] : 0.0f;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(&tmem_holder)),
                     "r"(kNetTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);   // the producer's expect_tx arrival + the copies' bytes
            mbar_init(&empty[s], 1);  // the MMA commit of the stage's tile
        }
        for (int b = 0; b < kNetBufs; ++b) {
            mbar_init(&tfull[b], 2);              // the MMA commit + the issuer's arrival (tile number)
            mbar_init(&tempty[b], kNetGroupWarps);  // one arrival per warp of the tile's group
        }
        mbar_init(&wbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_holder;

    if (warp == kNetEpiWarps) {
        // ---------------- producer: tiles blockIdx.x, + gridDim.x, ... in increasing order ----------------
        if (lane == 0) {
            mbar_expect_tx(&wbar, (uint32_t)net_weight_bytes(L));
            for (int l = 1; l < L; ++l) {
                const size_t off = (size_t)(l - 1) * kNetWHidden;
                bulk_g2s(sW + off, reinterpret_cast<const unsigned char *>(q.wtc) + off,
                         l < L - 1 ? kNetWHidden : kNetWLast, &wbar);
            }
        }
        const unsigned int need = (unsigned int)S;  // one release per tile of the row
        const int G = (int)gridDim.x;
        int ready = 0;  // tiles from this one on whose input rows are known complete
        int k = 0;
        for (;; ++k) {
            const int s = k % NS;
            int item = (int)blockIdx.x + k * G;
            if (item >= total) item = -1;
            Item it{};
            if (item >= 0) {
                if (lane == 0) trace_at(q, item, 0);
                it = decode(item, q.B, T, S);
                if (ready == 0) ready = net_deps(q, item, G, total, T, S, need, lane);
                if (ready == 0) item = -1;
                else --ready;
            }
            if (lane == 0) {
                if (item >= 0) trace_at(q, item, 1);
                // the stage's previous tile (k - NS) has been read by its MMAs, so its phase of
                // full[s] is complete (also before an end marker's arrival); if that wait runs
                // out, nothing more arrives on full[s] and the issuer's own wait runs out
                bool free = true;
                if (k >= NS && !mbar_wait(&empty[s], (uint32_t)((k / NS - 1) & 1))) {
                    atomicExch(q.err, 1);
                    item = -1;
                    free = false;
                }
                info[s] = item;
                if (item < 0) {
                    if (free) mbar_arrive(&full[s]);  // end marker
                } else {
                    trace_at(q, item, 2);
                    fence_proxy_async_global();
                    mbar_expect_tx(&full[s], (uint32_t)kNetHaloTx);
                    // padded rows t TR .. t TR + TR + 1 of strip xs: one contiguous run
                    const unsigned char *src = reinterpret_cast<const unsigned char *>(q.act[(it.l - 1) & 1]) +
                                               (((size_t)it.b * S + it.xs) * (q.H + 2) + (size_t)it.t * TR) * ROWB;
                    bulk_g2s(sStage + (size_t)s * kNetStage, src, (uint32_t)kNetHaloTx, &full[s]);
                    trace_at(q, item, 3);
                }
            }
            if (__shfl_sync(0xffffffffu, item, 0) < 0) break;
        }
        if (lane == 0) {
            // copies still in flight: the last fill of each stage, and the weights (bounded waits)
            for (int kk = (k - NS + 1 > 0 ? k - NS + 1 : 0); kk < k; ++kk)
                mbar_wait(&full[kk % NS], (uint32_t)((kk / NS) & 1));
            mbar_wait(&wbar, 0);
        }
        __syncwarp();
    } else if (warp == kNetEpiWarps + 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            bool ok = mbar_wait(&wbar, 0);
            if (!ok) atomicExch(q.err, 1);
            const uint32_t w0 = saddr(sW), st0 = saddr(sStage);
            const int per_layer = q.B * T * S;
            int k = 0, last_k = -1;
            for (;; ++k) {
                const int s = k % NS, bb = k % kNetBufs;
                int item = -1;
                if (ok) {
                    if (mbar_wait(&full[s], (uint32_t)((k / NS) & 1))) {
                        item = info[s];
                        if (item >= 0) trace_at(q, item, 4);
                    } else {
                        atomicExch(q.err, 1);
                        ok = false;
                    }
                }
                // the accumulator buffer's previous tile (k - 4) has been read by its epilogue
                // group, so its phase of tfull[bb] is complete (also before an end marker's
                // arrivals); if that wait runs out, nothing more arrives and the group's own wait
                // runs out
                if (k >= kNetBufs && !mbar_wait(&tempty[bb], (uint32_t)((k / kNetBufs - 1) & 1))) {
                    atomicExch(q.err, 1);
                    break;
                }
                tinfo[bb] = item;
                if (item < 0) {
                    // end markers for both epilogue groups (tiles k and k + 1)
                    mbar_arrive(&tfull[bb], 2);
                    const int k1 = k + 1, b1 = k1 % kNetBufs;
                    if (k1 < kNetBufs || mbar_wait(&tempty[b1], (uint32_t)((k1 / kNetBufs - 1) & 1))) {
                        tinfo[b1] = -1;
                        mbar_arrive(&tfull[b1], 2);
                    } else {
                        atomicExch(q.err, 1);
                    }
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const int l = 1 + item / per_layer;
                const uint32_t a0 = st0 + (uint32_t)(s * kNetStage), b0 = w0 + (uint32_t)((l - 1) * kNetWHidden);
                const uint32_t d0 = tmem + (uint32_t)(bb * TR * C);
                if (l == L - 1)
                    issue_conv_tile<16>(d0, a0, b0);
                else
                    issue_conv_tile<32>(d0, a0, b0);
                mma_commit(&empty[s]);   // the stage may be refilled once these MMAs are done
                mma_commit(&tfull[bb]);  // the accumulator is complete once these MMAs are done
                trace_at(q, item, 5);
                mbar_arrive(&tfull[bb]);
                last_k = k;
            }
            // MMAs still in flight: the last tile's commit (bounded wait)
            if (last_k >= 0) mbar_wait(&empty[last_k % NS], (uint32_t)((last_k / NS) & 1));
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: two groups of 8 warps take alternate tiles; in a group, warp
        // w reads lanes 32 (w % 4) .. + 31 (pixels) x 32 columns (channels) of tile row (w / 4) % 2
        const int grp = warp / kNetGroupWarps, qd = warp & 3, rr = (warp >> 2) & 1;
        for (int k = grp;; k += 2) {
            const int bb = k % kNetBufs;
            const bool got = mbar_wait(&tfull[bb], (uint32_t)((k / kNetBufs) & 1));
            if (!group_all(got, grp)) {  // a wait ran out: the whole group stops
                if (lane == 0) atomicExch(q.err, 1);
                break;
            }
            const int item = tinfo[bb];  // the same for the whole group
            if (item < 0) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const bool tr = (warp % kNetGroupWarps) == 0 && lane == 0;
            if (tr) trace_at(q, item, 6);
            const Item it = decode(item, q.B, T, S);
            const int y = it.t * TR + rr, x = it.xs * TM + qd * 32 + lane;
            const uint32_t taddr = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(bb * TR * C);
            if (it.l < L - 1) {
                uint32_t r[32];
                tmem_ld32(taddr + (uint32_t)(C * rr), r);
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[bb]);
                if (tr) trace_at(q, item, 7);
                uint4 v[4];
                gelu_chunks(r, sbias[it.l], v);
                store_px(q.act[it.l & 1], it.b, q.H, q.W, y, x, v);
                if (tr) trace_at(q, item, 8);
                net_release(q, 1 + (int)(((size_t)(it.l - 1) * q.B + it.b) * T + it.t), grp, tr);
            } else {
                uint32_t r0;
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n"
                             : "=r"(r0)
                             : "r"(taddr + (uint32_t)(16 * rr)));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[bb]);
                if (tr) trace_at(q, item, 7);
                q.yf[((size_t)it.b * q.H + y) * q.W + x] = (__uint_as_float(r0) + sbias[it.l][0]) * q.out_scale;
                if (tr) trace_at(q, item, 8);
            }
            if (tr) trace_at(q, item, 9);
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kNetTmemCols));
    // the last CTA to finish resets the counters for the next launch
    if (tid == 0) {
        __threadfence();
        s_last = (atomicAdd(q.sync, 1u) == gridDim.x - 1) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        const size_t n = net_sync_words(L, q.B, q.H);
        for (size_t i = tid; i < n; i += kNetThreads) q.sync[i] = 0u;
    }
}

}  // namespace

int net_stages_that_fit(int L)
{
    if (L < 3 || L > kNetMaxLayers) return 0;
    int dev = 0, optin = 0;
    cudaFuncAttributes fa{};
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, k_cnn_net) != cudaSuccess)
        return 0;
    for (int s = kNetMaxStages; s >= 2; --s)
        if (net_smem_bytes(L, s) + fa.sharedSizeBytes <= (size_t)optin) return s;
    return 0;
}

// One CTA per SM (the shared memory holds one), no more than there are tiles; a cooperative
// launch, which the driver refuses rather than run with CTAs that are not all resident.
cudaError_t net_launch(const NetLaunch &q_in, cudaStream_t stream, int *grid_out)
{
    NetLaunch q = q_in;
    cudaError_t e;
    const size_t smem = net_smem_bytes(q.L, q.stages);
    if ((e = cudaFuncSetAttribute(k_cnn_net, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cnn_net, kNetThreads, smem)) != cudaSuccess)
        return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const long long items = (long long)(q.L - 1) * q.B * (q.H / TR) * (q.W / TM);
    const int grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, items));
    if (grid_out) *grid_out = grid;
    void *args[] = {&q};
    return cudaLaunchCooperativeKernel((void *)k_cnn_net, grid, kNetThreads, args, smem, stream);
}

}  // namespace cnntc
}  // namespace dns2d
