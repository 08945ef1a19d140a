// psod_sort.cu -- device-wide exclusive scan and stable LSD radix sort.
//
// Both are plain HBM-bound passes: the scan reads and writes 4 B per
// element in three passes (tile reduce, tile-sum scan, tile scan + offset);
// the radix sort makes one histogram pass and one stable scatter pass per
// 8-bit digit, skipping digits that every key shares.
#include "psod_internal.cuh"

namespace psod {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ unsigned warp_incl_scan(unsigned v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// block-wide exclusive scan for blockDim.x <= 1024 (multiple of 32)
__device__ unsigned block_excl_scan(unsigned v, unsigned *total) {
  __shared__ unsigned s_warp[33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  unsigned inc = warp_incl_scan(v);
  if (lane == 31) s_warp[w] = inc;
  __syncthreads();
  if (w == 0) {
    unsigned x = lane < nw ? s_warp[lane] : 0u;
    unsigned xi = warp_incl_scan(x);
    if (lane < nw) s_warp[lane] = xi - x;
    if (lane == 31) s_warp[32] = xi;  // lanes >= nw add 0, so this is the total
  }
  __syncthreads();
  unsigned off = s_warp[w];
  unsigned tot = s_warp[32];
  __syncthreads();
  if (total) *total = tot;
  return off + inc - v;
}

__global__ void k_tile_reduce(const unsigned *in, long long n, unsigned *partial) {
  long long base = (long long)blockIdx.x * SCAN_TILE;
  unsigned s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  // reduce
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ unsigned sw[32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned v = threadIdx.x < (blockDim.x >> 5) ? sw[threadIdx.x] : 0u;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// per-tile exclusive scan; blocked layout (thread t owns items t*ITEMS..)
__global__ void k_tile_scan(const unsigned *in, unsigned *out, long long n, const unsigned *offsets,
                            unsigned *total_out) {
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  unsigned v[SCAN_ITEMS];
  unsigned s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    long long i = base + k;
    v[k] = (i < n) ? in[i] : 0u;
    s += v[k];
  }
  unsigned tot;
  unsigned ex = block_excl_scan(s, &tot);
  unsigned off = (offsets ? offsets[blockIdx.x] : 0u) + ex;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    long long i = base + k;
    if (i < n) out[i] = off;
    off += v[k];
  }
  if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) {
    // off now holds the inclusive sum through the last element of the tile
    *total_out = off;
  }
}

}  // namespace

static int scan_level(psod_ctx *c, const unsigned *in, unsigned *out, long long n, bool with_total, int level) {
  if (n <= 0) {
    if (with_total) PSOD_CUDA(c, cudaMemsetAsync(out, 0, sizeof(unsigned), c->stream));
    return PSOD_OK;
  }
  long long ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  unsigned *partial = nullptr;
  if (ntiles > 1) {
    // tile sums live in context scratch (slots 8.., one per recursion level)
    int st = scratch(c, 8 + level, (size_t)ntiles + 1, &partial);
    if (st) return st;
    k_tile_reduce<<<(unsigned)ntiles, SCAN_THREADS, 0, c->stream>>>(in, n, partial);
    st = scan_level(c, partial, partial, ntiles, false, level + 1);
    if (st) return st;
  }
  k_tile_scan<<<(unsigned)ntiles, SCAN_THREADS, 0, c->stream>>>(in, out, n, partial,
                                                                 with_total ? out + n : nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_check(c, e, "scan_u32");
  return PSOD_OK;
}

int scan_u32(psod_ctx *c, const unsigned *in, unsigned *out, long long n, bool with_total) {
  return scan_level(c, in, out, n, with_total, 0);
}

// ---------------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------------
namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_RADIX = 256;

// digit counts of a tile; lanes with equal digits are counted together
// (the top digits of clustered keys are shared by most of a tile)
template <typename K>
__global__ void k_radix_hist(const K *keys, long long n, int shift, unsigned *hist, long long ntiles) {
  __shared__ unsigned s_h[RS_RADIX];
  s_h[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  long long base = (long long)blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int k = 0; k < RS_ITEMS; k++) {
    const long long i = base + (long long)k * RS_THREADS + threadIdx.x;
    const bool valid = i < n;
    const unsigned d = valid ? ((unsigned)(keys[i] >> shift) & 0xffu) : (RS_RADIX + lane);
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(&s_h[d], (unsigned)__popc(peers));
  }
  __syncthreads();
  hist[(long long)threadIdx.x * ntiles + blockIdx.x] = s_h[threadIdx.x];
}

// Stable scatter.  Warp w of a tile owns its keys [w*512, (w+1)*512) and
// ranks them 32 at a time in input order (match_any on the digit, running
// per-warp digit counters); one scan over the warps per digit then gives
// each warp's start within the tile's digit run, and a scan over the digits
// each digit run's start within the tile.  The tile is first ordered by
// digit in shared memory, then written out by consecutive threads, so each
// digit run of the tile leaves as contiguous, coalesced stores (written
// straight from the ranking, a warp's 32 stores would hit up to 32 runs).
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_PER_LANE = RS_TILE / RS_THREADS;

template <typename K>
constexpr size_t rs_smem_bytes() {
  return (size_t)RS_TILE * (sizeof(K) + sizeof(unsigned));
}

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const K *keys, const unsigned *vals, K *okeys,
                                                              unsigned *ovals, long long n, int shift,
                                                              const unsigned *offsets, long long ntiles) {
  extern __shared__ __align__(16) unsigned char rs_smem[];
  K *sk = reinterpret_cast<K *>(rs_smem);                     // the tile's keys in digit order
  unsigned *sv = reinterpret_cast<unsigned *>(sk + RS_TILE);  // and their values
  __shared__ unsigned s_cnt[RS_WARPS][RS_RADIX];
  __shared__ unsigned s_base[RS_RADIX], s_loc[RS_RADIX];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
#pragma unroll
  for (int q = 0; q < RS_WARPS; q++) s_cnt[q][t] = 0;
  s_base[t] = offsets[(long long)t * ntiles + blockIdx.x];
  __syncthreads();
  const long long tile0 = (long long)blockIdx.x * RS_TILE;
  const long long base = tile0 + (long long)w * (32 * RS_PER_LANE);
  const unsigned lt = (1u << lane) - 1u;
  K k[RS_PER_LANE];
  unsigned v[RS_PER_LANE], rk[RS_PER_LANE];
  // all loads first (independent, in flight together), then the ranking
#pragma unroll
  for (int r = 0; r < RS_PER_LANE; r++) {
    const long long i = base + r * 32 + lane;
    const bool valid = i < n;
    k[r] = valid ? keys[i] : (K)0;
    v[r] = valid ? vals[i] : 0u;
  }
#pragma unroll
  for (int r = 0; r < RS_PER_LANE; r++) {
    const long long i = base + r * 32 + lane;
    const bool valid = i < n;
    const unsigned d = valid ? ((unsigned)(k[r] >> shift) & 0xffu) : (RS_RADIX + lane);
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    unsigned prev = 0;
    if (valid && lane == leader) {
      prev = s_cnt[w][d];
      s_cnt[w][d] = prev + __popc(peers);
    }
    prev = __shfl_sync(0xffffffffu, prev, leader);
    rk[r] = prev + __popc(peers & lt);
  }
  __syncthreads();
  {
    unsigned run = 0;
#pragma unroll
    for (int q = 0; q < RS_WARPS; q++) {
      const unsigned cnt = s_cnt[q][t];
      s_cnt[q][t] = run;
      run += cnt;
    }
    // run = the tile's count of digit t; its run starts at the exclusive sum
    s_loc[t] = block_excl_scan(run, nullptr);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_PER_LANE; r++) {
    const long long i = base + r * 32 + lane;
    if (i < n) {
      const unsigned d = (unsigned)(k[r] >> shift) & 0xffu;
      const unsigned p = s_loc[d] + s_cnt[w][d] + rk[r];  // < RS_TILE
      sk[p] = k[r];
      sv[p] = v[r];
    }
  }
  __syncthreads();
  const unsigned tile_n = (unsigned)min((long long)RS_TILE, n - tile0);
  for (unsigned j = t; j < tile_n; j += RS_THREADS) {
    const K key = sk[j];
    const unsigned d = (unsigned)(key >> shift) & 0xffu;
    const unsigned pos = s_base[d] + (j - s_loc[d]);
    okeys[pos] = key;
    ovals[pos] = sv[j];
  }
}

template <typename K>
__global__ void k_key_range(const K *keys, long long n, unsigned long long *mn_mx) {
  unsigned long long mn = ~0ull, mx = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long k = (unsigned long long)keys[i];
    mn = k < mn ? k : mn;
    mx = k > mx ? k : mx;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_down_sync(0xffffffffu, mn, o), b = __shfl_down_sync(0xffffffffu, mx, o);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mn_mx[0], mn);
    atomicMax(&mn_mx[1], mx);
  }
}

template <typename K>
int radix_sort_impl(psod_ctx *c, K *keys, unsigned *vals, long long n, int end_bit) {
  if (n <= 1) return PSOD_OK;
  // digits every key shares need no pass: find the highest differing bit
  unsigned long long *d_rng = nullptr;
  int st = scratch(c, SLOT_SORT_RNG, 2, &d_rng);
  if (st) return st;
  unsigned long long init[2] = {~0ull, 0ull};
  PSOD_CUDA(c, cudaMemcpyAsync(d_rng, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  k_key_range<K><<<592, 256, 0, c->stream>>>(keys, n, d_rng);
  unsigned long long rng[2] = {0, ~0ull};
  PSOD_CUDA(c, cudaMemcpyAsync(rng, d_rng, sizeof(rng), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  unsigned long long diff = rng[0] ^ rng[1];
  if (diff == 0) return PSOD_OK;  // all keys equal: a stable sort is the identity
  int hi_bit = 64 - __builtin_clzll(diff);
  if (hi_bit > end_bit) hi_bit = end_bit;
  int ndigits = (hi_bit + 7) / 8;
  long long ntiles = (n + RS_TILE - 1) / RS_TILE;
  K *tk = nullptr;
  unsigned *tv = nullptr, *hist = nullptr;
  if ((st = scratch(c, SLOT_SORT_KEYS, (size_t)n, &tk))) return st;
  if ((st = scratch(c, SLOT_SORT_VALS, (size_t)n, &tv))) return st;
  if ((st = scratch(c, SLOT_SORT_HIST, (size_t)ntiles * RS_RADIX + 1, &hist))) return st;
  PSOD_CUDA(c, cudaFuncSetAttribute(k_radix_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)rs_smem_bytes<K>()));
  K *ka = keys, *kb = tk;
  unsigned *va = vals, *vb = tv;
  for (int dgt = 0; dgt < ndigits; dgt++) {
    int shift = dgt * 8;
    k_radix_hist<K><<<(unsigned)ntiles, RS_THREADS, 0, c->stream>>>(ka, n, shift, hist, ntiles);
    st = scan_u32(c, hist, hist, ntiles * RS_RADIX, false);
    if (st) break;
    k_radix_scatter<K><<<(unsigned)ntiles, RS_THREADS, rs_smem_bytes<K>(), c->stream>>>(ka, va, kb, vb, n, shift,
                                                                                       hist, ntiles);
    K *tkk = ka;
    ka = kb;
    kb = tkk;
    unsigned *tvv = va;
    va = vb;
    vb = tvv;
  }
  if (!st && ka != keys) {
    cudaMemcpyAsync(keys, ka, sizeof(K) * n, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(vals, va, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, c->stream);
  }
  cudaError_t e = cudaGetLastError();
  cudaStreamSynchronize(c->stream);
  if (st) return st;
  if (e != cudaSuccess) return cuda_check(c, e, "radix_sort");
  return PSOD_OK;
}

}  // namespace

int radix_sort_u64(psod_ctx *c, unsigned long long *keys, unsigned *vals, long long n, int end_bit) {
  return radix_sort_impl<unsigned long long>(c, keys, vals, n, end_bit);
}
int radix_sort_u32(psod_ctx *c, unsigned *keys, unsigned *vals, long long n, int end_bit) {
  return radix_sort_impl<unsigned>(c, keys, vals, n, end_bit);
}

}  // namespace psod
