// Learned radius bracket: a small MLP that predicts, for each seed, the
// radius of the first ball the crossing search (k_cross) visits.
//
// The crossing search grows a ball around the refined centre until the
// Delta stop lies inside it; every ball that turns out too small costs a
// pass over its cells, and a ball much larger than needed costs a larger
// sort.  The network maps ten seed-local features (densities, shell counts
// from the per-cell alive table, the refinement sum, the centre offset) to
//   y0 = log(largest stop radius over the thresholds, in cells)
//   y1 = log(N_delta)
// and the search starts at exp(y0) times a margin.  A miss falls back to the
// growing search, so the halo table never depends on the network.
//
// Network: 10 (padded to 16) -> 64 -> 64 -> 2 (padded to 8), ReLU, BF16
// operands with FP32 accumulation on the tensor cores (mma.sync m16n8k16),
// FP32 master weights and Adam.  Rounding points (each also made by the
// test's numpy restatement): X = bf16((x - mu)/sigma); H1 = bf16(relu(X W1^T
// + b1)); H2 = bf16(relu(H1 W2^T + b2)); Y = H2 W3^T + b3 (FP32);
// dY = bf16((Y - T)/B); dH2 = bf16(dY W3 * [H2 > 0]); dH1 = bf16(dH2 W2 *
// [H1 > 0]); weight gradients dY^T H2, dH2^T H1, dH1^T X and bias gradients
// the column sums of dY, dH2, dH1, all accumulated in FP32.
//
// The whole network is 5,768 parameters and runs a few microseconds per
// scheduler round, so the warp-level mma.sync form (operands straight from
// shared memory, no tensor-memory allocation or descriptors) is used.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "psod_internal.cuh"

namespace psod {

namespace {

constexpr int NF = PSOD_LEARN_FEATURES;  // real features
constexpr int IN = 16;                   // padded input width
constexpr int HID = 64;                  // hidden width
constexpr int NOUT = 2;                  // outputs
constexpr int OUTP = 8;                  // padded output width
constexpr int TILE = 64;                 // samples per CTA, 16 per warp
constexpr int LTPB = 128;                // threads per CTA

// FP32 parameter layout (bf16 copies use the same matrix shapes)
constexpr int OW1 = 0;
constexpr int OB1 = OW1 + HID * IN;
constexpr int OW2 = OB1 + HID;
constexpr int OB2 = OW2 + HID * HID;
constexpr int OW3 = OB2 + HID;
constexpr int OB3 = OW3 + OUTP * HID;
constexpr int NPARAM = OB3 + OUTP;
// model blob: mu_x[16], sigma_x[16], mu_y[2], sigma_y[2], params
constexpr int NNORM = 2 * IN + 2 * NOUT;
constexpr int NBLOB = NNORM + NPARAM;
static_assert(NBLOB == PSOD_LEARN_MODEL_FLOATS, "model blob size");
static_assert(NPARAM == PSOD_LEARN_PARAMS, "parameter count");

typedef __nv_bfloat16 bf16;

// bf16 weight copies: row-major W1 [64][16], W2 [64][64], W3 [8][64], and
// transposes W2T [64][64] (W2T[i][o] = W2[o][i]), W3T [64][16] (o < 8)
struct Bf16W {
  bf16 w1[HID * IN];
  bf16 w2[HID * HID];
  bf16 w3[OUTP * HID];
  bf16 w2t[HID * HID];
  bf16 w3t[HID * IN];
};

struct Norm {
  float mux[IN], sgx[IN], muy[NOUT], sgy[NOUT];
};

// ---------------------------------------------------------------------------
// warp-level tensor-core tiles (m16n8k16, bf16 in, f32 accumulate)
// A: 16 rows x 16 k of a row-major bf16 matrix.  B: given as Bt, the
// row-major matrix whose row n is column n of B.  Accumulator element e of a
// lane sits at row (lane >> 2) + 8 * (e >> 1), column 2 * (lane & 3) + (e & 1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma16816(float c[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ unsigned ld2(const bf16 *p) { return *reinterpret_cast<const unsigned *>(p); }

__device__ __forceinline__ void load_a(unsigned a[4], const bf16 *A, int lda, int r0, int k0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const bf16 *p0 = A + (r0 + g) * lda + k0 + 2 * t;
  const bf16 *p1 = p0 + 8 * lda;
  a[0] = ld2(p0);
  a[1] = ld2(p1);
  a[2] = ld2(p0 + 8);
  a[3] = ld2(p1 + 8);
}

__device__ __forceinline__ void load_b(unsigned b[2], const bf16 *Bt, int ldb, int n0, int k0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const bf16 *p = Bt + (n0 + g) * ldb + k0 + 2 * t;
  b[0] = ld2(p);
  b[1] = ld2(p + 8);
}

// C[16 x 8*NT] = A[r0.., 0..16*KT) * B[.., n0..n0+8*NT)
template <int NT, int KT>
__device__ __forceinline__ void warp_gemm(float (&c)[NT][4], const bf16 *A, int lda, int r0, const bf16 *Bt, int ldb,
                                          int n0 = 0) {
#pragma unroll
  for (int j = 0; j < NT; j++) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
  for (int kt = 0; kt < KT; kt++) {
    unsigned a[4];
    load_a(a, A, lda, r0, kt * 16);
#pragma unroll
    for (int j = 0; j < NT; j++) {
      unsigned b[2];
      load_b(b, Bt, ldb, n0 + j * 8, kt * 16);
      mma16816(c[j], a, b);
    }
  }
}

__device__ __forceinline__ int frag_row(int e) { return ((threadIdx.x & 31) >> 2) + ((e >> 1) << 3); }
__device__ __forceinline__ int frag_col(int e) { return ((threadIdx.x & 3) << 1) + (e & 1); }

// shared-memory layout of the training and inference CTAs
struct LSmem {
  Bf16W w;
  float b1[HID], b2[HID], b3[OUTP];
  bf16 x[TILE * IN], xt[IN * TILE];
  bf16 h1[TILE * HID], h1t[HID * TILE];
  bf16 h2[TILE * HID], h2t[HID * TILE];
  bf16 dy[TILE * IN], dyt[IN * TILE];
  bf16 dh2[TILE * HID], dh2t[HID * TILE], dh1t[HID * TILE];
};

__device__ void load_weights(LSmem &S, const Bf16W *gw, const float *params) {
  const unsigned *src = reinterpret_cast<const unsigned *>(gw);
  unsigned *dst = reinterpret_cast<unsigned *>(&S.w);
  for (int i = threadIdx.x; i < (int)(sizeof(Bf16W) / 4); i += blockDim.x) dst[i] = src[i];
  for (int i = threadIdx.x; i < HID; i += blockDim.x) {
    S.b1[i] = params[OB1 + i];
    S.b2[i] = params[OB2 + i];
  }
  for (int i = threadIdx.x; i < OUTP; i += blockDim.x) S.b3[i] = params[OB3 + i];
}

// forward of the warp's 16 rows; y: the output tile (16 x 8, FP32).
// with_t: also write the transposed copies the backward pass needs
__device__ void forward_rows(LSmem &S, int r0, bool with_t, float (&y)[1][4]) {
  float c[8][4];
  warp_gemm<8, 1>(c, S.x, IN, r0, S.w.w1, IN);
#pragma unroll
  for (int j = 0; j < 8; j++)
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int r = r0 + frag_row(e), col = j * 8 + frag_col(e);
      const bf16 h = __float2bfloat16_rn(fmaxf(__fadd_rn(c[j][e], S.b1[col]), 0.f));
      S.h1[r * HID + col] = h;
      if (with_t) S.h1t[col * TILE + r] = h;
    }
  __syncwarp();
  warp_gemm<8, 4>(c, S.h1, HID, r0, S.w.w2, HID);
#pragma unroll
  for (int j = 0; j < 8; j++)
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int r = r0 + frag_row(e), col = j * 8 + frag_col(e);
      const bf16 h = __float2bfloat16_rn(fmaxf(__fadd_rn(c[j][e], S.b2[col]), 0.f));
      S.h2[r * HID + col] = h;
      if (with_t) S.h2t[col * TILE + r] = h;
    }
  __syncwarp();
  warp_gemm<1, 4>(y, S.h2, HID, r0, S.w.w3, HID);
#pragma unroll
  for (int e = 0; e < 4; e++) y[0][e] = __fadd_rn(y[0][e], S.b3[frag_col(e)]);
}

// sum over the 8 row groups of a warp (lanes with equal lane & 3)
__device__ __forceinline__ float rowgroup_sum(float v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  return v;
}

// One training tile: rows [base, base + TILE) of the batch.  Adds the
// gradient of 0.5 * sum (y - t)^2 / bsz over the tile into grad, and the
// tile's sum of squared errors into *sse.
__global__ void __launch_bounds__(LTPB) k_mlp_grad(const bf16 *X, const float *T, const unsigned *perm,
                                                   long long off, int bsz, const Bf16W *gw, const float *params,
                                                   float *grad, float *sse) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LSmem &S = *reinterpret_cast<LSmem *>(smem_raw);
  const int base = blockIdx.x * TILE;
  load_weights(S, gw, params);
  for (int i = threadIdx.x; i < TILE * IN; i += blockDim.x) {
    const int r = i / IN, k = i % IN;
    bf16 v = __float2bfloat16_rn(0.f);
    if (base + r < bsz) v = X[(size_t)perm[off + base + r] * IN + k];
    S.x[r * IN + k] = v;
    S.xt[k * TILE + r] = v;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, r0 = w * 16;
  float y[1][4];
  forward_rows(S, r0, true, y);
  // dY = (y - t) / bsz on the two real outputs of valid rows
  float loss = 0.f;
  const float inv_b = 1.0f / (float)bsz;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int r = r0 + frag_row(e), col = frag_col(e);
    float d = 0.f;
    if (col < NOUT && base + r < bsz) {
      const float diff = __fsub_rn(y[0][e], T[(size_t)perm[off + base + r] * NOUT + col]);
      loss = __fmaf_rn(diff, diff, loss);
      d = __fmul_rn(diff, inv_b);
    }
    const bf16 db = __float2bfloat16_rn(d);
    S.dy[r * IN + col] = db;
    S.dy[r * IN + col + 8] = __float2bfloat16_rn(0.f);
    S.dyt[col * TILE + r] = db;
    S.dyt[(col + 8) * TILE + r] = __float2bfloat16_rn(0.f);
    y[0][e] = __bfloat162float(db);
  }
  // bias 3
#pragma unroll
  for (int e = 0; e < 2; e++) {
    const float s = rowgroup_sum(y[0][e] + y[0][e + 2]);
    if ((threadIdx.x & 31) < 4 && frag_col(e) < NOUT) atomicAdd(&grad[OB3 + frag_col(e)], s);
  }
  loss = rowgroup_sum(loss);
  loss += __shfl_xor_sync(0xffffffffu, loss, 1);
  loss += __shfl_xor_sync(0xffffffffu, loss, 2);
  if ((threadIdx.x & 31) == 0) atomicAdd(sse, loss);
  __syncwarp();
  // dH2 = bf16(dY W3 * [H2 > 0])
  float c[8][4];
  warp_gemm<8, 1>(c, S.dy, IN, r0, S.w.w3t, IN);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float bs[2] = {0.f, 0.f};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int r = r0 + frag_row(e), col = j * 8 + frag_col(e);
      const float v = __bfloat162float(S.h2[r * HID + col]) > 0.f ? c[j][e] : 0.f;
      const bf16 d = __float2bfloat16_rn(v);
      S.dh2[r * HID + col] = d;
      S.dh2t[col * TILE + r] = d;
      bs[e & 1] += __bfloat162float(d);
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const float s = rowgroup_sum(bs[q]);
      if ((threadIdx.x & 31) < 4) atomicAdd(&grad[OB2 + j * 8 + frag_col(q)], s);
    }
  }
  __syncwarp();
  // dH1 = bf16(dH2 W2 * [H1 > 0])
  warp_gemm<8, 4>(c, S.dh2, HID, r0, S.w.w2t, HID);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float bs[2] = {0.f, 0.f};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int r = r0 + frag_row(e), col = j * 8 + frag_col(e);
      const float v = __bfloat162float(S.h1[r * HID + col]) > 0.f ? c[j][e] : 0.f;
      const bf16 d = __float2bfloat16_rn(v);
      S.dh1t[col * TILE + r] = d;
      bs[e & 1] += __bfloat162float(d);
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const float s = rowgroup_sum(bs[q]);
      if ((threadIdx.x & 31) < 4) atomicAdd(&grad[OB1 + j * 8 + frag_col(q)], s);
    }
  }
  __syncthreads();
  // weight gradients over the tile's samples (K = TILE); warp w owns the
  // output-feature rows [16w, 16w + 16)
  {
    float g2[8][4];
    warp_gemm<8, 4>(g2, S.dh2t, TILE, r0, S.h1t, TILE);
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int e = 0; e < 4; e++)
        atomicAdd(&grad[OW2 + (r0 + frag_row(e)) * HID + j * 8 + frag_col(e)], g2[j][e]);
    float g1[2][4];
    warp_gemm<2, 4>(g1, S.dh1t, TILE, r0, S.xt, TILE);
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int e = 0; e < 4; e++)
        atomicAdd(&grad[OW1 + (r0 + frag_row(e)) * IN + j * 8 + frag_col(e)], g1[j][e]);
    // W3: rows o < 2 of dY^T H2; warp w takes columns [16w, 16w + 16)
    float g3[2][4];
    warp_gemm<2, 4>(g3, S.dyt, TILE, 0, S.h2t, TILE, w * 16);
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int o = frag_row(e);
        if (o < NOUT) atomicAdd(&grad[OW3 + o * HID + w * 16 + j * 8 + frag_col(e)], g3[j][e]);
      }
  }
}

// Adam on the FP32 master parameters (bias-corrected moments)
__global__ void k_adam(float *p, float *m, float *v, const float *g, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// bf16 copies and transposes of the weights
__global__ void k_weights_bf16(const float *p, Bf16W *w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < HID * IN) {
    w->w1[i] = __float2bfloat16_rn(p[OW1 + i]);
    const int r = i / IN, o = i % IN;  // W3T[r][o] = W3[o][r], zero for o >= 8
    w->w3t[i] = __float2bfloat16_rn(o < OUTP ? p[OW3 + o * HID + r] : 0.f);
  }
  if (i < HID * HID) {
    w->w2[i] = __float2bfloat16_rn(p[OW2 + i]);
    const int o = i / HID, c = i % HID;
    w->w2t[c * HID + o] = __float2bfloat16_rn(p[OW2 + i]);
  }
  if (i < OUTP * HID) w->w3[i] = __float2bfloat16_rn(p[OW3 + i]);
}

// standardised bf16 inputs (rows padded to 16) and FP32 targets
__global__ void k_standardize(const float *x, const float *t, long long n, Norm nm, bf16 *X, float *T) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int k = 0; k < IN; k++) {
    const float v = k < NF ? __fdiv_rn(__fsub_rn(x[i * NF + k], nm.mux[k]), nm.sgx[k]) : 0.f;
    X[i * IN + k] = __float2bfloat16_rn(v);
  }
  if (t) {
#pragma unroll
    for (int k = 0; k < NOUT; k++) T[i * NOUT + k] = __fdiv_rn(__fsub_rn(t[i * NOUT + k], nm.muy[k]), nm.sgy[k]);
  }
}

// Forward pass of raw feature rows (row stride `stride`).  out: y in
// original units (2 per row) when rb0 is null; else rb0[i] = exp(y0)*margin,
// or 0 (no prediction) for rows whose column 15 is set (stride 16 only).
__global__ void __launch_bounds__(LTPB) k_mlp_forward(const float *x, int stride, long long n, Norm nm,
                                                      const Bf16W *gw, const float *params, float *out,
                                                      float *rb0, float margin) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LSmem &S = *reinterpret_cast<LSmem *>(smem_raw);
  const long long base = (long long)blockIdx.x * TILE;
  load_weights(S, gw, params);
  for (int i = threadIdx.x; i < TILE * IN; i += blockDim.x) {
    const int r = i / IN, k = i % IN;
    float v = 0.f;
    if (base + r < n && k < NF) v = __fdiv_rn(__fsub_rn(x[(base + r) * stride + k], nm.mux[k]), nm.sgx[k]);
    S.x[r * IN + k] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, r0 = w * 16;
  float y[1][4];
  forward_rows(S, r0, false, y);
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const long long r = base + r0 + frag_row(e);
    const int col = frag_col(e);
    if (r >= n || col >= NOUT) continue;
    const float v = __fmaf_rn(y[0][e], nm.sgy[col], nm.muy[col]);
    if (rb0) {
      if (col == 0) rb0[r] = x[r * stride + IN - 1] != 0.f ? 0.f : expf(v) * margin;
    } else {
      out[r * NOUT + col] = v;
    }
  }
}

size_t lsmem() { return sizeof(LSmem); }

}  // namespace

struct LearnState {
  bool has_model = false;
  Norm norm{};
  float *d_params = nullptr, *d_m = nullptr, *d_v = nullptr, *d_grad = nullptr, *d_sse = nullptr;
  Bf16W *d_w = nullptr;
  // collected samples
  bool collect = false;
  unsigned long long cap = 0;
  float *d_x = nullptr, *d_t = nullptr;
  unsigned long long *d_count = nullptr;
  float margin = 1.1f;
  bool attr_set = false;  // shared-memory attribute of the inference kernel
};

static int learn_alloc(psod_ctx *c) {
  if (!c->learn) c->learn = new LearnState();
  LearnState &L = *c->learn;
  if (L.d_params) return PSOD_OK;
  if (cudaMalloc(&L.d_params, sizeof(float) * NPARAM) != cudaSuccess ||
      cudaMalloc(&L.d_m, sizeof(float) * NPARAM) != cudaSuccess ||
      cudaMalloc(&L.d_v, sizeof(float) * NPARAM) != cudaSuccess ||
      cudaMalloc(&L.d_grad, sizeof(float) * NPARAM) != cudaSuccess ||
      cudaMalloc(&L.d_sse, sizeof(float)) != cudaSuccess || cudaMalloc(&L.d_w, sizeof(Bf16W)) != cudaSuccess) {
    cudaGetLastError();
    return set_err(c, PSOD_ERR_NOMEM, "learned bracket: device allocation failed");
  }
  return PSOD_OK;
}

void learn_free(psod_ctx *c) {
  if (!c->learn) return;
  LearnState &L = *c->learn;
  void *ptrs[] = {L.d_params, L.d_m, L.d_v, L.d_grad, L.d_sse, L.d_w, L.d_x, L.d_t, L.d_count};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete c->learn;
  c->learn = nullptr;
}

bool learn_ready(const psod_ctx *c) { return c->learn && c->learn->has_model; }
bool learn_collecting(const psod_ctx *c) { return c->learn && c->learn->collect; }

void learn_sample_buffers(const psod_ctx *c, float **x, float **t, unsigned long long **count,
                          unsigned long long *cap) {
  const LearnState &L = *c->learn;
  *x = L.d_x;
  *t = L.d_t;
  *count = L.d_count;
  *cap = L.cap;
}

int learn_predict(psod_ctx *c, const float *feat, unsigned n, float *rb0) {
  if (n == 0) return PSOD_OK;
  LearnState &L = *c->learn;
  if (!L.attr_set) {
    PSOD_CUDA(c, cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem()));
    L.attr_set = true;
  }
  k_mlp_forward<<<(n + TILE - 1) / TILE, LTPB, lsmem(), c->stream>>>(feat, IN, n, L.norm, L.d_w, L.d_params, nullptr,
                                                                      rb0, L.margin);
  PSOD_CUDA(c, cudaGetLastError());
  return PSOD_OK;
}

static int refresh_bf16(psod_ctx *c) {
  LearnState &L = *c->learn;
  k_weights_bf16<<<(HID * HID + 255) / 256, 256, 0, c->stream>>>(L.d_params, L.d_w);
  PSOD_CUDA(c, cudaGetLastError());
  return PSOD_OK;
}

static int set_model_blob(psod_ctx *c, const float *blob) {
  int st;
  if ((st = learn_alloc(c))) return st;
  LearnState &L = *c->learn;
  Norm nm{};
  memcpy(nm.mux, blob, sizeof(float) * IN);
  memcpy(nm.sgx, blob + IN, sizeof(float) * IN);
  memcpy(nm.muy, blob + 2 * IN, sizeof(float) * NOUT);
  memcpy(nm.sgy, blob + 2 * IN + NOUT, sizeof(float) * NOUT);
  for (int k = 0; k < IN; k++)
    if (!(nm.sgx[k] > 0.f)) return set_err(c, PSOD_ERR_ARG, "model: feature scales must be positive");
  for (int k = 0; k < NOUT; k++)
    if (!(nm.sgy[k] > 0.f)) return set_err(c, PSOD_ERR_ARG, "model: target scales must be positive");
  L.norm = nm;
  PSOD_CUDA(c, cudaMemcpyAsync(L.d_params, blob + NNORM, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, c->stream));
  if ((st = refresh_bf16(c))) return st;
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  L.has_model = true;
  return PSOD_OK;
}

}  // namespace psod

using namespace psod;

extern "C" {

int psod_learn_collect(psod_ctx *c, int64_t capacity) {
  if (!c) return PSOD_ERR_ARG;
  if (capacity < 0) return set_err(c, PSOD_ERR_ARG, "capacity must be >= 0");
  cudaSetDevice(c->device);
  int st;
  if ((st = learn_alloc(c))) return st;
  LearnState &L = *c->learn;
  if (capacity == 0) {
    L.collect = false;
    return PSOD_OK;
  }
  if ((unsigned long long)capacity != L.cap) {
    if (L.d_x) cudaFree(L.d_x);
    if (L.d_t) cudaFree(L.d_t);
    L.d_x = L.d_t = nullptr;
    L.cap = 0;
    if (cudaMalloc(&L.d_x, sizeof(float) * NF * capacity) != cudaSuccess ||
        cudaMalloc(&L.d_t, sizeof(float) * NOUT * capacity) != cudaSuccess) {
      cudaGetLastError();
      return set_err(c, PSOD_ERR_NOMEM, "sample buffer allocation failed");
    }
    L.cap = (unsigned long long)capacity;
  }
  if (!L.d_count && cudaMalloc(&L.d_count, sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return set_err(c, PSOD_ERR_NOMEM, "sample counter allocation failed");
  }
  PSOD_CUDA(c, cudaMemsetAsync(L.d_count, 0, sizeof(unsigned long long), c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  L.collect = true;
  return PSOD_OK;
}

int psod_learn_samples(psod_ctx *c, int64_t *n, float *x_out, float *t_out) {
  if (!c || !n) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  *n = 0;
  if (!c->learn || !c->learn->d_count) return PSOD_OK;
  LearnState &L = *c->learn;
  unsigned long long cnt = 0;
  PSOD_CUDA(c, cudaMemcpyAsync(&cnt, L.d_count, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  cnt = std::min(cnt, L.cap);
  *n = (int64_t)cnt;
  int st;
  if (x_out && cnt && (st = copy_out(c, x_out, L.d_x, sizeof(float) * NF * cnt))) return st;
  if (t_out && cnt && (st = copy_out(c, t_out, L.d_t, sizeof(float) * NOUT * cnt))) return st;
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  return PSOD_OK;
}

int psod_learn_set_model(psod_ctx *c, const float *blob, int64_t nfloats) {
  if (!c || !blob) return PSOD_ERR_ARG;
  if (nfloats != NBLOB) return set_err(c, PSOD_ERR_ARG, "model blob has the wrong size");
  cudaSetDevice(c->device);
  std::vector<float> h(NBLOB);
  if (is_device_ptr(blob)) {
    PSOD_CUDA(c, cudaMemcpy(h.data(), blob, sizeof(float) * NBLOB, cudaMemcpyDeviceToHost));
  } else {
    memcpy(h.data(), blob, sizeof(float) * NBLOB);
  }
  return set_model_blob(c, h.data());
}

int psod_learn_get_model(psod_ctx *c, float *blob, int64_t nfloats) {
  if (!c || !blob) return PSOD_ERR_ARG;
  if (nfloats != NBLOB) return set_err(c, PSOD_ERR_ARG, "model blob has the wrong size");
  if (!learn_ready(c)) return set_err(c, PSOD_ERR_STATE, "no model: train or set one first");
  cudaSetDevice(c->device);
  LearnState &L = *c->learn;
  std::vector<float> h(NBLOB);
  memcpy(h.data(), L.norm.mux, sizeof(float) * IN);
  memcpy(h.data() + IN, L.norm.sgx, sizeof(float) * IN);
  memcpy(h.data() + 2 * IN, L.norm.muy, sizeof(float) * NOUT);
  memcpy(h.data() + 2 * IN + NOUT, L.norm.sgy, sizeof(float) * NOUT);
  PSOD_CUDA(c, cudaMemcpyAsync(h.data() + NNORM, L.d_params, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost,
                               c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  if (is_device_ptr(blob)) {
    PSOD_CUDA(c, cudaMemcpy(blob, h.data(), sizeof(float) * NBLOB, cudaMemcpyHostToDevice));
  } else {
    memcpy(blob, h.data(), sizeof(float) * NBLOB);
  }
  return PSOD_OK;
}

int psod_learn_set_margin(psod_ctx *c, float margin) {
  if (!c) return PSOD_ERR_ARG;
  if (!(margin >= 1.0f)) return set_err(c, PSOD_ERR_ARG, "margin must be >= 1");
  cudaSetDevice(c->device);
  int st;
  if ((st = learn_alloc(c))) return st;
  c->learn->margin = margin;
  return PSOD_OK;
}

int psod_learn_forward(psod_ctx *c, int64_t n, const float *x, float *y) {
  if (!c || n < 0 || (n > 0 && (!x || !y))) return PSOD_ERR_ARG;
  if (!learn_ready(c)) return set_err(c, PSOD_ERR_STATE, "no model: train or set one first");
  if (n == 0) return PSOD_OK;
  cudaSetDevice(c->device);
  LearnState &L = *c->learn;
  float *dx = nullptr, *dy = nullptr;
  int st;
  if ((st = scratch(c, SLOT_LEARN_X, (size_t)n * NF, &dx)) || (st = scratch(c, SLOT_LEARN_Y, (size_t)n * NOUT, &dy)))
    return st;
  if ((st = copy_in(c, dx, x, sizeof(float) * NF * n))) return st;
  PSOD_CUDA(c, cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem()));
  k_mlp_forward<<<(unsigned)((n + TILE - 1) / TILE), LTPB, lsmem(), c->stream>>>(dx, NF, n, L.norm, L.d_w,
                                                                                  L.d_params, dy, nullptr, 1.f);
  PSOD_CUDA(c, cudaGetLastError());
  if ((st = copy_out(c, y, dy, sizeof(float) * NOUT * n))) return st;
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  return PSOD_OK;
}

int psod_learn_gradient(psod_ctx *c, int64_t n, const float *x, const float *t, float *grad, float *loss_out) {
  if (!c) return PSOD_ERR_ARG;
  if (n <= 0 || n > (1 << 20) || !x || !t || !grad) return set_err(c, PSOD_ERR_ARG, "gradient: need 1..2^20 rows");
  if (!learn_ready(c)) return set_err(c, PSOD_ERR_STATE, "no model: train or set one first");
  cudaSetDevice(c->device);
  LearnState &L = *c->learn;
  float *dx = nullptr, *dt = nullptr, *tstd = nullptr;
  bf16 *xb = nullptr;
  unsigned *perm = nullptr;
  int st;
  if ((st = scratch(c, SLOT_LEARN_X, (size_t)n * NF, &dx)) || (st = scratch(c, SLOT_LEARN_Y, (size_t)n * NOUT, &dt)) ||
      (st = scratch(c, SLOT_LEARN_XB, (size_t)n * IN, &xb)) ||
      (st = scratch(c, SLOT_LEARN_TS, (size_t)n * NOUT, &tstd)) || (st = scratch(c, SLOT_LEARN_PERM, (size_t)n, &perm)))
    return st;
  if ((st = copy_in(c, dx, x, sizeof(float) * NF * n)) || (st = copy_in(c, dt, t, sizeof(float) * NOUT * n)))
    return st;
  std::vector<unsigned> id((size_t)n);
  for (int64_t i = 0; i < n; i++) id[(size_t)i] = (unsigned)i;
  PSOD_CUDA(c, cudaMemcpyAsync(perm, id.data(), sizeof(unsigned) * n, cudaMemcpyHostToDevice, c->stream));
  k_standardize<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(dx, dt, n, L.norm, xb, tstd);
  PSOD_CUDA(c, cudaMemsetAsync(L.d_grad, 0, sizeof(float) * NPARAM, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(L.d_sse, 0, sizeof(float), c->stream));
  PSOD_CUDA(c, cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem()));
  k_mlp_grad<<<(unsigned)((n + TILE - 1) / TILE), LTPB, lsmem(), c->stream>>>(xb, tstd, perm, 0, (int)n, L.d_w,
                                                                              L.d_params, L.d_grad, L.d_sse);
  PSOD_CUDA(c, cudaGetLastError());
  if ((st = copy_out(c, grad, L.d_grad, sizeof(float) * NPARAM))) return st;
  float sse = 0.f;
  PSOD_CUDA(c, cudaMemcpyAsync(&sse, L.d_sse, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  if (loss_out) *loss_out = 0.5f * sse / (float)n;
  return PSOD_OK;
}

int psod_learn_train(psod_ctx *c, const psod_train_params *tp, float *loss_out) {
  if (!c || !tp) return PSOD_ERR_ARG;
  if (tp->epochs < 1 || tp->batch < TILE || tp->batch % TILE || !(tp->lr > 0.f))
    return set_err(c, PSOD_ERR_ARG, "train: epochs >= 1, batch a multiple of 64, lr > 0");
  cudaSetDevice(c->device);
  int st;
  int64_t n = 0;
  if ((st = psod_learn_samples(c, &n, nullptr, nullptr))) return st;
  if (n < 2 * TILE) return set_err(c, PSOD_ERR_STATE, "train: fewer than 128 collected samples");
  if (n > (int64_t)0xffffffffll) return set_err(c, PSOD_ERR_ARG, "train: too many samples");
  if ((st = learn_alloc(c))) return st;
  LearnState &L = *c->learn;
  // feature and target scales (host, double accumulation)
  std::vector<float> hx((size_t)n * NF), ht((size_t)n * NOUT);
  if ((st = psod_learn_samples(c, &n, hx.data(), ht.data()))) return st;
  Norm nm{};
  for (int k = 0; k < IN; k++) {
    nm.mux[k] = 0.f;
    nm.sgx[k] = 1.f;
  }
  auto stats = [&](const std::vector<float> &a, int stride, int k, float &mu, float &sg) {
    double s = 0, s2 = 0;
    for (int64_t i = 0; i < n; i++) {
      const double v = a[(size_t)i * stride + k];
      s += v;
      s2 += v * v;
    }
    const double m = s / n, var = std::max(s2 / n - m * m, 0.0);
    mu = (float)m;
    sg = (float)std::max(std::sqrt(var), 1e-6);
  };
  for (int k = 0; k < NF; k++) stats(hx, NF, k, nm.mux[k], nm.sgx[k]);
  for (int k = 0; k < NOUT; k++) stats(ht, NOUT, k, nm.muy[k], nm.sgy[k]);
  L.norm = nm;
  // initial weights: uniform(+-sqrt(6/fan_in)) on the real inputs; zero
  // padding and biases
  std::vector<float> p(NPARAM, 0.f);
  std::mt19937_64 rng(tp->seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  const float a1 = std::sqrt(6.f / NF), a2 = std::sqrt(6.f / HID), a3 = std::sqrt(6.f / HID) * 0.5f;
  for (int o = 0; o < HID; o++)
    for (int i = 0; i < NF; i++) p[OW1 + o * IN + i] = a1 * u(rng);
  for (int i = 0; i < HID * HID; i++) p[OW2 + i] = a2 * u(rng);
  for (int o = 0; o < NOUT; o++)
    for (int i = 0; i < HID; i++) p[OW3 + o * HID + i] = a3 * u(rng);
  PSOD_CUDA(c, cudaMemcpyAsync(L.d_params, p.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(L.d_m, 0, sizeof(float) * NPARAM, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(L.d_v, 0, sizeof(float) * NPARAM, c->stream));
  if ((st = refresh_bf16(c))) return st;
  // standardised data set
  bf16 *xb = nullptr;
  float *tstd = nullptr;
  unsigned *perm = nullptr;
  if ((st = scratch(c, SLOT_LEARN_XB, (size_t)n * IN, &xb)) ||
      (st = scratch(c, SLOT_LEARN_TS, (size_t)n * NOUT, &tstd)) || (st = scratch(c, SLOT_LEARN_PERM, (size_t)n, &perm)))
    return st;
  k_standardize<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(L.d_x, L.d_t, n, nm, xb, tstd);
  PSOD_CUDA(c, cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem()));
  const float b1 = tp->beta1 > 0.f ? tp->beta1 : 0.9f, b2 = tp->beta2 > 0.f ? tp->beta2 : 0.999f;
  const float eps = tp->eps > 0.f ? tp->eps : 1e-8f;
  std::vector<unsigned> order((size_t)n);
  for (int64_t i = 0; i < n; i++) order[(size_t)i] = (unsigned)i;
  long long step = 0;
  for (int e = 0; e < tp->epochs; e++) {
    std::shuffle(order.begin(), order.end(), rng);
    PSOD_CUDA(c, cudaMemcpyAsync(perm, order.data(), sizeof(unsigned) * n, cudaMemcpyHostToDevice, c->stream));
    PSOD_CUDA(c, cudaMemsetAsync(L.d_sse, 0, sizeof(float), c->stream));
    for (int64_t off = 0; off < n; off += tp->batch) {
      const int bsz = (int)std::min<int64_t>(tp->batch, n - off);
      PSOD_CUDA(c, cudaMemsetAsync(L.d_grad, 0, sizeof(float) * NPARAM, c->stream));
      k_mlp_grad<<<(unsigned)((bsz + TILE - 1) / TILE), LTPB, lsmem(), c->stream>>>(xb, tstd, perm, off, bsz, L.d_w,
                                                                                    L.d_params, L.d_grad, L.d_sse);
      step++;
      const float c1 = 1.f - (float)std::pow((double)b1, (double)step);
      const float c2 = 1.f - (float)std::pow((double)b2, (double)step);
      k_adam<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(L.d_params, L.d_m, L.d_v, L.d_grad, NPARAM, tp->lr, b1,
                                                          b2, eps, c1, c2);
      if ((st = refresh_bf16(c))) return st;
    }
    PSOD_CUDA(c, cudaGetLastError());
    float sse = 0.f;
    PSOD_CUDA(c, cudaMemcpyAsync(&sse, L.d_sse, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    if (loss_out) loss_out[e] = 0.5f * sse / (float)n;
  }
  L.has_model = true;
  return PSOD_OK;
}

}  // extern "C"
