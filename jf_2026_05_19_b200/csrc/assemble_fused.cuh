// assemble_fused.cuh -- persistent CQUAD4 + block-reduction kernel.
//
// The separate path writes every staged CQUAD4 block to HBM (q4_k_kernel)
// and reads it back in a second kernel (block_reduce1_kernel): 2.9 GB each
// way per K assembly of a 0.9M-CQUAD4 mesh, far beyond the 126 MB L2.  This
// kernel runs both as tasks of one persistent launch, in chunk order, so
// that a block is summed while its staged slots are still in L2:
//
//   * the CQUAD4s are cut into chunks of consecutive elements (a multiple of
//     24, so that whole CTA tiles of either width fit); each block's
//     completion chunk is the last chunk holding one of its CQUAD4 pairs;
//   * the task list is R(-1), E(0), E(1), R(0), E(2), R(1), ... E(C-1),
//     R(C-2), R(C-1): E(c) = the CTA tiles of chunk c, R(c) = the blocks
//     completing at chunk c (R(-1): blocks without a CQUAD4 pair), in
//     CSC order, kFzRounds * W * 5 blocks per task;
//   * a CTA claims tasks from one atomic counter (the next claim is issued
//     while the current task runs).  After an E task the CTA publishes its
//     staging stores (barrier, then one thread's fence and an atomic add to
//     the chunk's done counter).  An R task of chunk c first waits until the
//     chunks c - span .. c are done (span = the widest chunk range of any
//     block's CQUAD4 pairs), then sums its blocks exactly as
//     block_reduce1_kernel does, reading staged values through L2.
//
// Progress: tasks are claimed in list order and an E task never waits, so
// every E task an R task waits for was claimed earlier by a CTA that is
// running it.  The wait is still bounded (kFzSpin polls); if it runs out the
// kernel sets the handle's error word, which the host reads back at its next
// synchronisation, and the call reports JFG_ERR_CUDA.
//
// Every block is summed in the same slot order by the same arithmetic as
// block_reduce1_kernel, so the values are bitwise those of the separate
// path.  CTRIA3 and bar tiles run before this kernel; their staged slots are
// read like the CQUAD4 ones.
//
// Included by jfg_api.cu inside its anonymous namespace, after the block
// reduction helpers and before the launch-shape attributes are set.

constexpr int kFzRounds = 2;         // block rounds per R task (5 blocks per warp per round)
constexpr int kFzSpin = 1 << 20;     // polls of a chunk counter before giving up (about 0.1-0.3 s)

struct FzArgs {
    const int4 *task = nullptr;      // (kind | chunk << 1, begin, end, first chunk to wait for)
    int64_t n_task = 0;
    const int32_t *order = nullptr;  // blocks in completion-chunk order
    const int32_t *need = nullptr;   // E tasks per chunk
    int *ctr = nullptr;              // [0] error word (sticky), [1] claim counter, [2 + c] done E tasks of chunk c
    int64_t nq = 0;
    const int32_t *nodes = nullptr;
    const double *prop = nullptr, *coords = nullptr, *nodeR = nullptr, *u = nullptr;
    double k6rot = 0.0;
    ElemOut o;
    const int32_t *seg = nullptr, *rot = nullptr, *slot_bar = nullptr;
    int64_t kg_rot_off = 0;
    const int64_t *pa = nullptr, *pb = nullptr;
    const int2 *len = nullptr;
    double *nz = nullptr;
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Blocks order[j0 .. j1) of an R task: warp w, lanes 6g .. 6g+5 take block
// j0 + 5 (w + W r) + g in round r; thread i sums row i, the rows meet in the
// warp's shared tile, and the two CSC writes follow block_reduce1_kernel.
template <bool KG, int W>
__device__ __forceinline__ void fz_reduce(const FzArgs &a, int64_t j0, int64_t j1, double *tr) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / 6, i = lane - 6 * (lane / 6);
    double *tile = tr + 36 * (5 * warp + (g < 5 ? g : 0));
    for (int64_t base = j0 + 5 * warp; base < j1; base += 5 * W) {
        const int64_t j = base + g;
        const bool one = g < 5 && j < j1;
        int64_t p_a = 0, p_b = -1;
        int2 l = make_int2(0, 0);
        if (one) {
            const int32_t k = __ldg(a.order + j);
            p_a = __ldg(a.pa + k);
            p_b = __ldg(a.pb + k);
            l = __ldg(a.len + k);
            const int32_t a0 = __ldg(a.seg + k), b0 = __ldg(a.seg + k + 1);
            if (KG) {
                const int32_t aa[1] = {a0}, bb[1] = {b0}, rr[1] = {__ldg(a.rot + k)};
                double *const tt[1] = {tile};
                block_kg_sums<1, true>(a.o.staging, a.o.staging + a.kg_rot_off, a.slot_bar, aa, rr, bb, i, tt);
            } else {
                double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                block_row_sum<true>(a.o.staging, a0, b0, i, s);
#pragma unroll
                for (int c = 0; c < 6; ++c) tile[6 * i + c] = s[c];
            }
        }
        __syncwarp();
        if (one) {
            const int64_t ca = p_a + i;
#pragma unroll
            for (int r = 0; r < 6; ++r) a.nz[ca + (int64_t)r * l.x] = tile[6 * r + i];
            if (p_b >= 0) {
                const int64_t cb = p_b + i;
#pragma unroll
                for (int c = 0; c < 6; ++c) a.nz[cb + (int64_t)c * l.y] = tile[6 * i + c];
            }
        }
        __syncwarp();  // the tile is rewritten in the next round
    }
}

template <bool KG, int W>
__device__ __forceinline__ void fz_body(const FzArgs &a, unsigned char *smem) {
    __shared__ int s_next[2];
    const int tid = threadIdx.x;
    if (tid == 0) s_next[0] = atomicAdd(a.ctr + 1, 1);
    __syncthreads();
    int buf = 0;
    for (int64_t t = s_next[0]; t < a.n_task;) {
        if (tid == 0) s_next[buf ^ 1] = atomicAdd(a.ctr + 1, 1);  // next claim, read after the barrier below
        const int4 tk = __ldg(a.task + t);
        if ((tk.x & 1) == 0) {
            const int c = tk.x >> 1;
            for (int64_t tile = tk.y; tile < tk.z; ++tile) {
                if (KG)
                    q4_kg_tile<W>(tile, reinterpret_cast<Q4GShared *>(smem), a.nq, a.nodes, a.prop, a.coords, a.nodeR, a.u, a.o);
                else
                    q4_k_tile<W>(tile, reinterpret_cast<Q4KShared *>(smem), a.nq, a.nodes, a.prop, a.coords, a.nodeR, a.k6rot, a.o);
                __syncwarp();
            }
            __syncthreads();  // every warp's staging stores are issued
            if (tid == 0) {
                __threadfence();
                atomicAdd(a.ctr + 2 + c, 1);
            }
        } else {
            const int c = (tk.x >> 1) - 1;  // -1: blocks without a CQUAD4 pair, ready at launch
            if (tid == 0 && c >= 0) {
                for (int cc = tk.w; cc <= c; ++cc) {
                    const int need = __ldg(a.need + cc);
                    for (int spin = 0; ld_acquire_gpu(a.ctr + 2 + cc) < need;) {
                        // give up after kFzSpin polls, or at once when another
                        // CTA already gave up (the error word is set)
                        if (++spin > kFzSpin || ((spin & 63) == 0 && ld_acquire_gpu(a.ctr) != 0)) {
                            atomicOr(a.ctr, 1);
                            break;
                        }
                        __nanosleep(100);
                    }
                }
                __threadfence();
            }
            __syncthreads();
            fz_reduce<KG, W>(a, tk.y, tk.z, reinterpret_cast<double *>(smem));
            __syncthreads();  // shared memory is reused by the next task
        }
        t = s_next[buf ^ 1];
        buf ^= 1;
    }
}

// Dynamic shared memory: the larger of the tile's element records and the
// reduction tiles (W * 5 blocks of 36 doubles).
template <int W>
__host__ __device__ constexpr size_t fz_smem_bytes(bool kg) {
    return (size_t)Q4_TEAMS_PER_WARP * W * (kg ? sizeof(Q4GShared) : sizeof(Q4KShared)) > (size_t)W * 5 * 36 * sizeof(double)
               ? (size_t)Q4_TEAMS_PER_WARP * W * (kg ? sizeof(Q4GShared) : sizeof(Q4KShared))
               : (size_t)W * 5 * 36 * sizeof(double);
}

template <int W>
__global__ void __launch_bounds__(32 * W, 16 / W) fused_k_kernel(FzArgs a) {
    extern __shared__ __align__(16) unsigned char fz_smem[];
    fz_body<false, W>(a, fz_smem);
}

template <int W>
__global__ void __launch_bounds__(32 * W, W == 4 ? 5 : 2) fused_kg_kernel(FzArgs a) {
    extern __shared__ __align__(16) unsigned char fz_smem[];
    fz_body<true, W>(a, fz_smem);
}

// Schedule build: per block, the first and last chunk holding one of its
// CQUAD4 pairs (RBE2-path pairs have no block).
__global__ void fz_chunk_kernel(int64_t nq, int64_t chunk, const int32_t *__restrict__ q4_slot, const int32_t *__restrict__ seg,
                                int64_t n_blk, int *cmin, int *cmax) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= 10 * nq) return;
    const int32_t sl = __ldg(q4_slot + x);
    if (sl < 0) return;
    const int32_t s = sl & kBlkIndexMask;
    int64_t lo = 0, hi = n_blk;  // last block k with seg[k] <= s
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(seg + mid) <= s) lo = mid;
        else hi = mid;
    }
    const int c = (int)((x / 10) / chunk);
    atomicMin(cmin + lo, c);
    atomicMax(cmax + lo, c);
}

// Sort key (completion chunk + 1), the block index, the per-key counts and
// the widest chunk range.
__global__ void fz_key_kernel(int64_t n_blk, const int *__restrict__ cmin, const int *__restrict__ cmax, int32_t *key,
                              int32_t *idx, int *count, int *span) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_blk) return;
    const int hi = cmax[k];
    key[k] = hi + 1;
    idx[k] = (int32_t)k;
    atomicAdd(count + hi + 1, 1);
    if (hi >= 0) atomicMax(span, hi - cmin[k]);
}
