// Learned preconditioner: a message-passing network over the matrix graph.
//
// No counterpart in the reference (it has no learned component); this is
// the learned part of the path, used inside flexible COCG with SSOR-COCG as
// the fallback.  Network (width H = 48, L = 6 layers, BF16 weights and
// activations, FP32 accumulation):
//   s_i = sqrt|A_ii|, rn = r / rms(r)
//   x_i = [Re rn_i/s_i, Im rn_i/s_i, K_ii/|A_ii|, omega M_ii/|A_ii|, bc_i, 1, 0, 0]
//   h0 = x W_in;  X_i = [h_i | sum_j a_ij h_j | sum_j b_ij h_j],
//   a_ij = K_ij/(s_i s_j), b_ij = omega M_ij/(s_i s_j)
//   h <- h + relu(X W_l + c_l)   (l = 0..5, GEMM 144 x 48 on the tensor cores)
//   z_i = r_i/s_i^2 + rms * (o_i0 + i o_i1)/s_i,  o = h W_out  (Jacobi term + learned correction)
// One fused kernel per layer: the block aggregates its 64 rows' neighbours (all rows
// at once, 2 lanes per row, 16-byte loads) into a shared-memory tile, with the
// message weights of every matrix entry computed once per solve, then every warp
// multiplies its 16 x 144 tile by W_l with
// mma.sync.m16n8k16 (BF16 in, FP32 accumulate) and applies bias, ReLU and the
// residual in registers.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "afem_internal.h"

namespace afem {

namespace mpnn {

constexpr int H = 48;
constexpr int L = 6;
constexpr int FIN = 8;
constexpr int XW = 3 * H;        // 144 columns of the layer input
constexpr int XS = XW + 8;       // padded shared-memory stride (bf16), conflict-free fragments
constexpr int ROWS = 64;         // rows per block (4 warps x 16)
constexpr int NPARAM = FIN * H + L * (XW * H + H) + H * 2;

// parameter offsets in the flat FP32 vector
__host__ __device__ constexpr int off_win() { return 0; }
__host__ __device__ constexpr int off_w(int l) { return FIN * H + l * (XW * H + H); }
__host__ __device__ constexpr int off_c(int l) { return off_w(l) + XW * H; }
__host__ __device__ constexpr int off_wout() { return FIN * H + L * (XW * H + H); }

}  // namespace mpnn

namespace {

using namespace mpnn;

__device__ __forceinline__ unsigned pack_bf16(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<unsigned*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(unsigned u) {
  __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162*>(&u);
  return __bfloat1622float2(v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Per-row scale s_i = sqrt|A_ii| and the static features, for one omega per system.
__global__ void k_rowinfo(const double2* __restrict__ km, const int32_t* __restrict__ diagpos,
                          const uint8_t* __restrict__ bc, int n, const double* __restrict__ omega, int ns,
                          float* __restrict__ s_out, float4* __restrict__ feat) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)n * ns) return;
  const int row = (int)(i % n), sy = (int)(i / n);
  const double2 d = km[diagpos[row]];
  const double om = omega[sy];
  const double ar = d.x, ai = om * d.y;
  const double mag = sqrt(ar * ar + ai * ai);
  s_out[i] = (float)sqrt(mag);
  feat[i] = make_float4((float)(ar / mag), (float)(ai / mag), bc ? (float)bc[row] : 0.f, 1.f);
}

// The message weights of every matrix entry for one omega per system, computed once per solve
// (every layer of every application reuses them): ew[sy*nnz + k] = (K_ij, omega M_ij)/(s_i s_j)
// for j != i, 0 on the diagonal (which the aggregation leaves out).
__global__ void k_edge_w(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                         const double2* __restrict__ km, const float* __restrict__ s,
                         const double* __restrict__ omega, int n, int ns, long nnz, float2* __restrict__ ew) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)n * ns) return;
  const int row = (int)(i % n), sy = (int)(i / n);
  const float si = s[i];
  const double om = omega[sy];
  float2* out = ew + (long)sy * nnz;
  for (int k = rowptr[row]; k < rowptr[row + 1]; ++k) {
    const int j = col[k];
    if (j == row) {
      out[k] = make_float2(0.f, 0.f);
      continue;
    }
    const double2 e = km[k];
    const float inv = 1.0f / (si * s[(long)sy * n + j]);
    out[k] = make_float2((float)e.x * inv, (float)(om * e.y) * inv);
  }
}

// h0 = x W_in (FP32 FMA, K = 8), rows x systems in one launch.
template <class V>
__global__ void k_encode(const V* __restrict__ r, int n, int ns, const float* __restrict__ s,
                         const float4* __restrict__ feat, const double* __restrict__ rms,
                         const float* __restrict__ win, __nv_bfloat16* __restrict__ h, const int* skip) {
  if (skip && *skip) return;
  __shared__ float w[FIN * H];
  for (int k = threadIdx.x; k < FIN * H; k += blockDim.x) w[k] = win[k];
  __syncthreads();
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)n * ns) return;
  const int row = (int)(i % n), sy = (int)(i / n);
  const V ri = r[(long)row * ns + sy];
  const float inv = (float)(1.0 / rms[sy]) / s[i];
  const float4 f = feat[i];
  const float x[FIN] = {(float)ri.x * inv, (float)ri.y * inv, f.x, f.y, f.z, f.w, 0.f, 0.f};
  unsigned* out = reinterpret_cast<unsigned*>(h + i * H);
  for (int c = 0; c < H; c += 2) {
    float a = 0.f, b = 0.f;
#pragma unroll
    for (int k = 0; k < FIN; ++k) {
      a += x[k] * w[k * H + c];
      b += x[k] * w[k * H + c + 1];
    }
    out[c / 2] = pack_bf16(a, b);
  }
}

// One message-passing layer for rows x systems (blockIdx.y = system).
// save_x / save_y (training) keep the layer input tile and the pre-activation.
__device__ __forceinline__ void agg_add(float (&aa)[24], float (&ab)[24], float2 w, const uint4 (&u)[3]) {
  const unsigned* q = reinterpret_cast<const unsigned*>(u);
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const float2 hj = unpack_bf16(q[k]);
    aa[2 * k] += w.x * hj.x; aa[2 * k + 1] += w.x * hj.y;
    ab[2 * k] += w.y * hj.x; ab[2 * k + 1] += w.y * hj.y;
  }
}

__global__ void __launch_bounds__(128)
    k_layer(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col, const float2* __restrict__ ew,
            long nnz, int n, const __nv_bfloat16* __restrict__ h_in, __nv_bfloat16* __restrict__ h_out,
            const __nv_bfloat16* __restrict__ wt,  // W_l transposed, bf16 [H][XW]
            const float* __restrict__ bias, __nv_bfloat16* __restrict__ save_x, __nv_bfloat16* __restrict__ save_y,
            const int* skip) {
  if (skip && *skip) return;
  __shared__ __align__(16) __nv_bfloat16 xs[ROWS * XS];
  __shared__ __align__(16) __nv_bfloat16 ws[H * XS];
  const int sy = blockIdx.y;
  const long base = (long)sy * n;
  for (int k = threadIdx.x; k < H * XW; k += blockDim.x) ws[(k / XW) * XS + (k % XW)] = wt[k];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = blockIdx.x * ROWS + w * 16;
  // ---- aggregate: all 64 rows of the block at once, two lanes per row, each lane owning
  // features 24*half .. 24*half+23 (three 16-byte words of the row's 96 bytes), two
  // neighbours' loads in flight; each feature sums its neighbours in entry order
  {
    const int rr = threadIdx.x >> 1, half = threadIdx.x & 1;
    const int row = blockIdx.x * ROWS + rr;
    unsigned* xrow = reinterpret_cast<unsigned*>(xs + rr * XS);
    if (row < n) {
      float aa[24], ab[24];
#pragma unroll
      for (int k = 0; k < 24; ++k) { aa[k] = 0.f; ab[k] = 0.f; }
      const uint4* own = reinterpret_cast<const uint4*>(h_in + (base + row) * H) + 3 * half;
      const uint4 o[3] = {own[0], own[1], own[2]};
      const float2* ewr = ew + (long)sy * nnz;
      const int k1 = rowptr[row + 1];
      int k = rowptr[row];
      for (; k + 1 < k1; k += 2) {
        const int ja = col[k], jb = col[k + 1];
        const float2 wa = ewr[k], wb = ewr[k + 1];
        const uint4* pa = reinterpret_cast<const uint4*>(h_in + (base + ja) * H) + 3 * half;
        const uint4* pb = reinterpret_cast<const uint4*>(h_in + (base + jb) * H) + 3 * half;
        const uint4 ua[3] = {pa[0], pa[1], pa[2]}, ub[3] = {pb[0], pb[1], pb[2]};
        agg_add(aa, ab, wa, ua);
        agg_add(aa, ab, wb, ub);
      }
      if (k < k1) {
        const int j = col[k];
        const float2 wj = ewr[k];
        const uint4* pj = reinterpret_cast<const uint4*>(h_in + (base + j) * H) + 3 * half;
        const uint4 uj[3] = {pj[0], pj[1], pj[2]};
        agg_add(aa, ab, wj, uj);
      }
      const unsigned* ow = reinterpret_cast<const unsigned*>(o);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        xrow[12 * half + q] = ow[q];
        xrow[24 + 12 * half + q] = pack_bf16(aa[2 * q], aa[2 * q + 1]);
        xrow[48 + 12 * half + q] = pack_bf16(ab[2 * q], ab[2 * q + 1]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        xrow[12 * half + q] = 0u;
        xrow[24 + 12 * half + q] = 0u;
        xrow[48 + 12 * half + q] = 0u;
      }
    }
  }
  __syncthreads();
  // ---- GEMM: rows 16w..16w+15 of the tile times W_l (XW x H)
  const int g = lane >> 2, t = lane & 3;
  float acc[6][4];
#pragma unroll
  for (int nt = 0; nt < 6; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
  const unsigned* X = reinterpret_cast<const unsigned*>(xs);
  const unsigned* W = reinterpret_cast<const unsigned*>(ws);
  constexpr int XSW = XS / 2;  // row stride in 32-bit words
#pragma unroll
  for (int ks = 0; ks < XW / 16; ++ks) {
    const int kw = ks * 8;  // word offset of column 16*ks
    unsigned a[4];
    a[0] = X[(w * 16 + g) * XSW + kw + t];
    a[1] = X[(w * 16 + g + 8) * XSW + kw + t];
    a[2] = X[(w * 16 + g) * XSW + kw + 4 + t];
    a[3] = X[(w * 16 + g + 8) * XSW + kw + 4 + t];
#pragma unroll
    for (int nt = 0; nt < 6; ++nt) {
      unsigned b[2];
      b[0] = W[(nt * 8 + g) * XSW + kw + t];
      b[1] = W[(nt * 8 + g) * XSW + kw + 4 + t];
      mma_bf16(acc[nt], a, b);
    }
  }
  // ---- epilogue: bias, relu, residual
#pragma unroll
  for (int nt = 0; nt < 6; ++nt) {
    const int c = nt * 8 + 2 * t;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int tr = w * 16 + g + half * 8;
      const int row = blockIdx.x * ROWS + tr;
      if (row >= n) continue;
      const float y0 = acc[nt][2 * half] + bias[c], y1 = acc[nt][2 * half + 1] + bias[c + 1];
      const float2 hv = unpack_bf16(X[tr * XSW + c / 2]);
      const long o = (base + row) * H + c;
      reinterpret_cast<unsigned*>(h_out + o)[0] = pack_bf16(hv.x + fmaxf(y0, 0.f), hv.y + fmaxf(y1, 0.f));
      if (save_y) reinterpret_cast<unsigned*>(save_y + o)[0] = pack_bf16(y0, y1);
    }
  }
  if (save_x) {
    for (int rr = 0; rr < 16; ++rr) {
      const int row = r0 + rr;
      if (row >= n) break;
      const unsigned* xrow = X + (w * 16 + rr) * XSW;
      unsigned* dst = reinterpret_cast<unsigned*>(save_x + (base + row) * XW);
      for (int q = lane; q < XW / 2; q += 32) dst[q] = xrow[q];
    }
  }
}

// z_i = r_i / s_i^2 + rms * (o0 + i o1) / s_i with o = h W_out.
template <class V>
__global__ void k_decode(const __nv_bfloat16* __restrict__ h, int n, int ns, const float* __restrict__ s,
                         const double* __restrict__ rms, const float* __restrict__ wout, const V* __restrict__ r,
                         V* __restrict__ z, float* __restrict__ o_save, const int* skip, int add) {
  if (skip && *skip) return;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)n * ns) return;
  const int row = (int)(i % n), sy = (int)(i / n);
  const unsigned* hv = reinterpret_cast<const unsigned*>(h + i * H);
  float o0 = 0.f, o1 = 0.f;
  for (int c = 0; c < H; c += 2) {
    const float2 v = unpack_bf16(hv[c / 2]);
    o0 += v.x * wout[c * 2] + v.y * wout[(c + 1) * 2];
    o1 += v.x * wout[c * 2 + 1] + v.y * wout[(c + 1) * 2 + 1];
  }
  if (o_save) {
    o_save[2 * i] = o0;
    o_save[2 * i + 1] = o1;
  }
  const float si = s[i];
  const float f = (float)rms[sy] / si, jac = 1.0f / (si * si);
  V out;
  if (add) {  // the correction on top of a base preconditioner's output already in z
    const V zi = z[(long)row * ns + sy];
    out.x = zi.x + o0 * f;
    out.y = zi.y + o1 * f;
  } else {
    const V ri = r[(long)row * ns + sy];
    out.x = o0 * f + (float)ri.x * jac;
    out.y = o1 * f + (float)ri.y * jac;
  }
  z[(long)row * ns + sy] = out;
}

// ------------------------------------------------------------------ training: loss
// res = A z - r and partial sums of |res|^2, |r|^2 (system sy = blockIdx.y, vectors [row][sys]).
__global__ void k_loss_res(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                           const double2* __restrict__ km, const double* __restrict__ omega, int n, int ns,
                           const double2* __restrict__ z, const double2* __restrict__ r, double2* __restrict__ res,
                           double* __restrict__ part) {
  const int sy = blockIdx.y;
  const double om = omega[sy];
  double a = 0.0, b = 0.0;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    double t1x = 0, t1y = 0, t2x = 0, t2y = 0;
    for (int k = rowptr[row]; k < rowptr[row + 1]; ++k) {
      const double2 e = km[k];
      const double2 zj = z[(long)col[k] * ns + sy];
      t1x += e.x * zj.x; t1y += e.x * zj.y;
      t2x += e.y * zj.x; t2y += e.y * zj.y;
    }
    const double2 ri = r[(long)row * ns + sy];
    const double2 q = make_double2(t1x - om * t2y - ri.x, t1y + om * t2x - ri.y);
    res[(long)row * ns + sy] = q;
    a += q.x * q.x + q.y * q.y;
    b += ri.x * ri.x + ri.y * ri.y;
  }
  for (int m = 16; m > 0; m >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, m);
    b += __shfl_xor_sync(0xffffffffu, b, m);
  }
  __shared__ double sa[32], sb[32];
  if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = a; sb[threadIdx.x >> 5] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { ta += sa[w]; tb += sb[w]; }
    part[((long)sy * gridDim.x + blockIdx.x) * 2] = ta;
    part[((long)sy * gridDim.x + blockIdx.x) * 2 + 1] = tb;
  }
}

__global__ void k_loss_sum(const double* __restrict__ part, int nb, int ns, double* __restrict__ out) {
  // out[2*sy] = sum |res|^2, out[2*sy+1] = sum |r|^2
  const int sy = threadIdx.x;
  if (sy >= ns) return;
  double a = 0, b = 0;
  for (int i = 0; i < nb; ++i) { a += part[((long)sy * nb + i) * 2]; b += part[((long)sy * nb + i) * 2 + 1]; }
  out[2 * sy] = a;
  out[2 * sy + 1] = b;
}

// dL/do: gz = 2 conj(A) res / |r|^2; do = (gz.re, gz.im) * rms / s  (FP32, system-major rows)
__global__ void k_loss_grad(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                            const double2* __restrict__ km, const double* __restrict__ omega, int n, int ns,
                            const double2* __restrict__ res, const double* __restrict__ sums,
                            const double* __restrict__ rms, const float* __restrict__ s, float* __restrict__ dout) {
  const int sy = blockIdx.y;
  const double om = omega[sy];
  const double f = 2.0 / sums[2 * sy + 1];
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    double t1x = 0, t1y = 0, t2x = 0, t2y = 0;
    for (int k = rowptr[row]; k < rowptr[row + 1]; ++k) {
      const double2 e = km[k];
      const double2 q = res[(long)col[k] * ns + sy];
      t1x += e.x * q.x; t1y += e.x * q.y;
      t2x += e.y * q.x; t2y += e.y * q.y;
    }
    // conj(A) q = K q - i omega M q
    const double gx = f * (t1x + om * t2y), gy = f * (t1y - om * t2x);
    const long i = (long)sy * n + row;
    const double sc = rms[sy] / (double)s[i];
    dout[2 * i] = (float)(gx * sc);
    dout[2 * i + 1] = (float)(gy * sc);
  }
}

// ------------------------------------------------------------------ training: backward
// dh = do W_out^T; dW_out += h^T do   (rows system-major; warp per row, lane = features 2l, 2l+1)
__global__ void k_decode_bwd(const __nv_bfloat16* __restrict__ h, long rows, const float* __restrict__ dout,
                             const float* __restrict__ wout, float* __restrict__ dh, float* __restrict__ gwout) {
  __shared__ float red[H * 2];
  for (int k = threadIdx.x; k < H * 2; k += blockDim.x) red[k] = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long warp = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * (long)blockDim.x) >> 5;
  float g00 = 0.f, g01 = 0.f, g10 = 0.f, g11 = 0.f;  // dW_out rows 2l, 2l+1, cols 0, 1
  const int c = 2 * lane;
  float w00 = 0.f, w01 = 0.f, w10 = 0.f, w11 = 0.f;
  if (lane < 24) { w00 = wout[c * 2]; w01 = wout[c * 2 + 1]; w10 = wout[(c + 1) * 2]; w11 = wout[(c + 1) * 2 + 1]; }
  for (long i = warp; i < rows; i += nw) {
    const float d0 = dout[2 * i], d1 = dout[2 * i + 1];
    if (lane < 24) {
      const float2 v = unpack_bf16(reinterpret_cast<const unsigned*>(h + i * H)[lane]);
      dh[i * H + c] = d0 * w00 + d1 * w01;
      dh[i * H + c + 1] = d0 * w10 + d1 * w11;
      g00 += v.x * d0; g01 += v.x * d1;
      g10 += v.y * d0; g11 += v.y * d1;
    }
  }
  if (lane < 24) {
    atomicAdd(&red[c * 2], g00); atomicAdd(&red[c * 2 + 1], g01);
    atomicAdd(&red[(c + 1) * 2], g10); atomicAdd(&red[(c + 1) * 2 + 1], g11);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < H * 2; k += blockDim.x) atomicAdd(&gwout[k], red[k]);
}

// Per 64-row tile: dY = dh * (Y > 0); dX = dY W^T (tensor cores); dW += X^T dY (tensor cores);
// dc += sum dY.  dX goes to global (the neighbour part is aggregated by k_agg_bwd).
__global__ void __launch_bounds__(128)
    k_layer_bwd(long rows, const float* __restrict__ dh, const __nv_bfloat16* __restrict__ sx,
                const __nv_bfloat16* __restrict__ sy_, const __nv_bfloat16* __restrict__ wl,  // W_l bf16 [XW][H]
                float* __restrict__ dx, float* __restrict__ gw, float* __restrict__ gc) {
  // dynamic shared memory (50.6 KB): dY tile [row][H], dY^T [H][row], X^T [XW][row], W_l [XW][H]
  constexpr int DS = H + 8, TS = ROWS + 8, WS = H + 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* dys = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  __nv_bfloat16* dyt = dys + ROWS * DS;
  __nv_bfloat16* xt = dyt + H * TS;
  __nv_bfloat16* wsm = xt + XW * TS;
  __shared__ float csum[H];
  const long r0 = (long)blockIdx.x * ROWS;
  for (int k = threadIdx.x; k < XW * H; k += blockDim.x) wsm[(k / H) * WS + (k % H)] = wl[k];
  if (threadIdx.x < H) csum[threadIdx.x] = 0.f;
  for (int k = threadIdx.x; k < ROWS * H; k += blockDim.x) {
    const int rr = k / H, c = k % H;
    const long row = r0 + rr;
    float v = 0.f;
    if (row < rows) {
      const float y = __bfloat162float(sy_[row * H + c]);
      v = y > 0.f ? dh[row * H + c] : 0.f;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    dys[rr * DS + c] = b;
    dyt[c * TS + rr] = b;
  }
  for (int k = threadIdx.x; k < ROWS * XW; k += blockDim.x) {
    const int rr = k / XW, c = k % XW;
    const long row = r0 + rr;
    xt[c * TS + rr] = (row < rows) ? sx[row * XW + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // dc
  for (int k = threadIdx.x; k < ROWS * H; k += blockDim.x)
    atomicAdd(&csum[k % H], __bfloat162float(dys[(k / H) * DS + (k % H)]));  // the tile's rows are padded to DS
  // ---- dX (rows 16w.. x XW) = dY (16 x H) * W^T: B[k=j][n=m] = W[m][j] -> [n][k] = wsm rows
  {
    const unsigned* A = reinterpret_cast<const unsigned*>(dys);
    const unsigned* B = reinterpret_cast<const unsigned*>(wsm);
    for (int nt = 0; nt < XW / 8; ++nt) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < H / 16; ++ks) {
        const int kw = ks * 8;
        unsigned a[4], b[2];
        a[0] = A[(w * 16 + g) * (DS / 2) + kw + t];
        a[1] = A[(w * 16 + g + 8) * (DS / 2) + kw + t];
        a[2] = A[(w * 16 + g) * (DS / 2) + kw + 4 + t];
        a[3] = A[(w * 16 + g + 8) * (DS / 2) + kw + 4 + t];
        b[0] = B[(nt * 8 + g) * (WS / 2) + kw + t];
        b[1] = B[(nt * 8 + g) * (WS / 2) + kw + 4 + t];
        mma_bf16(acc, a, b);
      }
      const int c = nt * 8 + 2 * t;
      for (int half = 0; half < 2; ++half) {
        const long row = r0 + w * 16 + g + half * 8;
        if (row < rows) {
          dx[row * XW + c] = acc[2 * half];
          dx[row * XW + c + 1] = acc[2 * half + 1];
        }
      }
    }
  }
  // ---- dW (XW x H) += X^T (XW x 64 rows) * dY (64 x H): A = xt [m][k], B[k][n] = dY[k][n] -> [n][k] = dyt
  {
    const unsigned* A = reinterpret_cast<const unsigned*>(xt);
    const unsigned* B = reinterpret_cast<const unsigned*>(dyt);
    for (int mt = w; mt < XW / 16; mt += 4) {
      for (int nt = 0; nt < H / 8; ++nt) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < ROWS / 16; ++ks) {
          const int kw = ks * 8;
          unsigned a[4], b[2];
          a[0] = A[(mt * 16 + g) * (TS / 2) + kw + t];
          a[1] = A[(mt * 16 + g + 8) * (TS / 2) + kw + t];
          a[2] = A[(mt * 16 + g) * (TS / 2) + kw + 4 + t];
          a[3] = A[(mt * 16 + g + 8) * (TS / 2) + kw + 4 + t];
          b[0] = B[(nt * 8 + g) * (TS / 2) + kw + t];
          b[1] = B[(nt * 8 + g) * (TS / 2) + kw + 4 + t];
          mma_bf16(acc, a, b);
        }
        const int m = mt * 16 + g, c = nt * 8 + 2 * t;
        atomicAdd(&gw[m * H + c], acc[0]);
        atomicAdd(&gw[m * H + c + 1], acc[1]);
        atomicAdd(&gw[(m + 8) * H + c], acc[2]);
        atomicAdd(&gw[(m + 8) * H + c + 1], acc[3]);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < H) atomicAdd(&gc[threadIdx.x], csum[threadIdx.x]);
}

constexpr size_t LAYER_BWD_SMEM = sizeof(__nv_bfloat16) * ((size_t)ROWS * (H + 8) + (size_t)H * (ROWS + 8) +
                                                           (size_t)XW * (ROWS + 8) + (size_t)XW * (H + 8));

// dh_prev = dh + dX[:, :H] + sum_j a_ij dX_j[H:2H] + sum_j b_ij dX_j[2H:3H]   (a, b symmetric)
__global__ void k_agg_bwd(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                          const double2* __restrict__ km, const float* __restrict__ s,
                          const double* __restrict__ omega, int n, const float* __restrict__ dx,
                          float* __restrict__ dh) {
  const int sy = blockIdx.y;
  const long base = (long)sy * n;
  const double om = omega[sy];
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int row = warp; row < n; row += nw) {
    const float si = s[base + row];
    float acc0 = 0.f, acc1 = 0.f;  // features lane, lane + 32 (< H)
    for (int k = rowptr[row]; k < rowptr[row + 1]; ++k) {
      const int j = col[k];
      if (j == row) continue;
      const double2 a = km[k];
      const float inv = 1.0f / (si * s[base + j]);
      const float wa = (float)a.x * inv, wb = (float)(om * a.y) * inv;
      const float* dj = dx + (base + j) * XW;
      acc0 += wa * dj[H + lane] + wb * dj[2 * H + lane];
      if (lane + 32 < H) acc1 += wa * dj[H + lane + 32] + wb * dj[2 * H + lane + 32];
    }
    const float* di = dx + (base + row) * XW;
    dh[(base + row) * H + lane] += di[lane] + acc0;
    if (lane + 32 < H) dh[(base + row) * H + lane + 32] += di[lane + 32] + acc1;
  }
}

// dW_in += x^T dh0 with x rebuilt from r (K = 8); warp per row, lane = features lane, lane + 32
template <class V>
__global__ void k_encode_bwd(const V* __restrict__ r, int n, int ns, const float* __restrict__ s,
                             const float4* __restrict__ feat, const double* __restrict__ rms,
                             const float* __restrict__ dh, float* __restrict__ gwin) {
  __shared__ float red[FIN * H];
  for (int k = threadIdx.x; k < FIN * H; k += blockDim.x) red[k] = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long warp = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * (long)blockDim.x) >> 5;
  float acc0[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, acc1[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (long i = warp; i < (long)n * ns; i += nw) {
    const int row = (int)(i % n), sy = (int)(i / n);
    const V ri = r[(long)row * ns + sy];
    const float inv = (float)(1.0 / rms[sy]) / s[i];
    const float4 f = feat[i];
    const float x[6] = {(float)ri.x * inv, (float)ri.y * inv, f.x, f.y, f.z, f.w};
    const float d0 = dh[i * H + lane];
    const float d1 = (lane + 32 < H) ? dh[i * H + lane + 32] : 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) { acc0[k] += x[k] * d0; acc1[k] += x[k] * d1; }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    atomicAdd(&red[k * H + lane], acc0[k]);
    if (lane + 32 < H) atomicAdd(&red[k * H + lane + 32], acc1[k]);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < FIN * H; k += blockDim.x) atomicAdd(&gwin[k], red[k]);
}

// Adam on the FP32 master weights (Kingma & Ba, 2015), then the BF16 copies.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ gsum, float* __restrict__ m1,
                       float* __restrict__ m2, int np, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       float gscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float g = gsum[i] * gscale;
  const float a = b1 * m1[i] + (1.f - b1) * g;
  const float b = b2 * m2[i] + (1.f - b2) * g * g;
  m1[i] = a;
  m2[i] = b;
  p[i] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

// BF16 copies of the layer weights: W_l as [XW][H] and transposed [H][XW]; FP32 copies of the small ones.
__global__ void k_cast_weights(const float* __restrict__ p, __nv_bfloat16* __restrict__ wl,
                               __nv_bfloat16* __restrict__ wt, float* __restrict__ small) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < L * XW * H) {
    const int l = i / (XW * H), k = i % (XW * H), m = k / H, c = k % H;
    const __nv_bfloat16 b = __float2bfloat16_rn(p[off_w(l) + k]);
    wl[i] = b;
    wt[l * XW * H + c * XW + m] = b;
  }
  // small: W_in (FIN*H), c_l (L*H), W_out (2H), bf16-rounded then widened
  const int ns = FIN * H + L * H + 2 * H;
  if (i < ns) {
    float v;
    if (i < FIN * H) v = __bfloat162float(__float2bfloat16_rn(p[off_win() + i]));
    else if (i < FIN * H + L * H) {
      const int l = (i - FIN * H) / H, c = (i - FIN * H) % H;
      v = p[off_c(l) + c];  // biases stay FP32
    } else v = __bfloat162float(__float2bfloat16_rn(p[off_wout() + (i - FIN * H - L * H)]));
    small[i] = v;
  }
}

}  // namespace

// ====================================================================== host side
struct MpnnState {
  DBuf<float> p, m1, m2, grad;           // FP32 master weights, Adam moments, gradient sum
  DBuf<__nv_bfloat16> wl, wt;            // BF16 layer weights [L][XW][H] and transposed [L][H][XW]
  DBuf<float> small;                     // W_in, biases, W_out (FP32, W_in/W_out BF16-rounded)
  bool cast_valid = false;
  int adam_t = 0;
  int base = 0;  // 0: z = r/|A_ii| + correction (Jacobi base); 1: z = H(r) + correction, H the gradient-corrected SSOR
  // workspace for n x ns rows
  long rows = 0;
  int ns = 0;
  DBuf<float> s;
  DBuf<float4> feat;
  DBuf<float2> ew;                       // message weights per (system, matrix entry), per solve
  DBuf<double> omega, rms;
  DBuf<__nv_bfloat16> h[L + 1];          // activations (training keeps all; inference ping-pongs 0/1)
  DBuf<__nv_bfloat16> sx[L], sy[L];      // saved layer inputs / pre-activations (training)
  DBuf<float> dh, dx, dout;
  DBuf<double2> z64, res, r64;
  DBuf<double> part, sums;
};

namespace {

MpnnState* state(afem_ctx* c) {
  if (!c->mpnn) c->mpnn = new MpnnState();
  return c->mpnn;
}

void ensure_cast(afem_ctx* c, MpnnState* S) {
  AFEM_REQUIRE(S->p.p, AFEM_ESTATE, "learned preconditioner: no weights loaded");
  if (S->cast_valid) return;
  S->wl.alloc((size_t)L * XW * H);
  S->wt.alloc((size_t)L * XW * H);
  S->small.alloc(FIN * H + L * H + 2 * H);
  k_cast_weights<<<(L * XW * H + 255) / 256, 256, 0, c->stream>>>(S->p.p, S->wl.p, S->wt.p, S->small.p);
  count_launch();
  S->cast_valid = true;
}

void ensure_work(afem_ctx* c, MpnnState* S, int ns, bool train) {
  const long rows = (long)c->nline * ns;
  if (S->rows != rows || S->ns != ns) {
    S->rows = rows;
    S->ns = ns;
    S->s.alloc(rows);
    S->feat.alloc(rows);
    S->omega.alloc(ns);
    S->rms.alloc(ns);
    for (int l = 0; l <= L; ++l) S->h[l].release();
    for (int l = 0; l < L; ++l) { S->sx[l].release(); S->sy[l].release(); }
    S->dh.release(); S->dx.release(); S->dout.release();
  }
  const int nh = train ? L + 1 : 2;
  for (int l = 0; l < nh; ++l) S->h[l].alloc((size_t)rows * H);
  if (train) {
    for (int l = 0; l < L; ++l) { S->sx[l].alloc((size_t)rows * XW); S->sy[l].alloc((size_t)rows * H); }
    S->dh.alloc((size_t)rows * H);
    S->dx.alloc((size_t)rows * XW);
    S->dout.alloc((size_t)rows * 2);
  }
}

unsigned blocks(long n, int t) { return (unsigned)((n + t - 1) / t); }

// Forward pass for ns systems. r, z: [row][sys]; rms[sy] and omega[sy] on the device.
void rowinfo(afem_ctx* c, MpnnState* S, int ns) {
  const long rows = (long)c->nline * ns;
  k_rowinfo<<<blocks(rows, 256), 256, 0, c->stream>>>(c->km.p, c->diagpos.p, c->bc.p, c->nline, S->omega.p, ns, S->s.p,
                                                       S->feat.p);
  count_launch();
  S->ew.alloc((size_t)ns * c->nnz);
  k_edge_w<<<blocks(rows, 128), 128, 0, c->stream>>>(c->rowptr.p, c->col.p, c->km.p, S->s.p, S->omega.p, c->nline, ns,
                                                     c->nnz, S->ew.p);
  count_launch();
}

template <class V>
void forward(afem_ctx* c, MpnnState* S, int ns, const V* r, V* z, bool train, const double* rms = nullptr,
             const int* skip = nullptr, int add = 0) {
  cudaStream_t st = c->stream;
  const int n = c->nline;
  const long rows = (long)n * ns;
  const double* R = rms ? rms : S->rms.p;
  k_encode<V><<<blocks(rows, 256), 256, 0, st>>>(r, n, ns, S->s.p, S->feat.p, R, S->small.p + 0, S->h[0].p, skip);
  count_launch();
  dim3 grid(blocks(n, ROWS), ns);
  for (int l = 0; l < L; ++l) {
    const __nv_bfloat16* hin = train ? S->h[l].p : S->h[l & 1].p;
    __nv_bfloat16* hout = train ? S->h[l + 1].p : S->h[(l + 1) & 1].p;
    k_layer<<<grid, 128, 0, st>>>(c->rowptr.p, c->col.p, S->ew.p, c->nnz, n, hin, hout,
                                  S->wt.p + (size_t)l * XW * H, S->small.p + FIN * H + l * H,
                                  train ? S->sx[l].p : nullptr, train ? S->sy[l].p : nullptr, skip);
    count_launch();
  }
  const __nv_bfloat16* hl = train ? S->h[L].p : S->h[L & 1].p;
  k_decode<V><<<blocks(rows, 256), 256, 0, st>>>(hl, n, ns, S->s.p, R, S->small.p + FIN * H + L * H, r, z,
                                                 nullptr, skip, add);
  count_launch();
  AFEM_CUDA(cudaGetLastError());
}

// Loss ||A z - r||^2/||r||^2 (summed over systems) and the gradient added to S->grad.
double loss_backward(afem_ctx* c, MpnnState* S, int ns, const double2* r) {
  cudaStream_t st = c->stream;
  const int n = c->nline;
  const long rows = (long)n * ns;
  S->z64.alloc(rows);
  S->res.alloc(rows);
  static bool attr_set = false;
  if (!attr_set) {
    AFEM_CUDA(cudaFuncSetAttribute(k_layer_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LAYER_BWD_SMEM));
    attr_set = true;
  }
  rowinfo(c, S, ns);
  if (S->base) {
    // z = H(r) + correction: the base preconditioner's output first, the network adds to it
    AFEM_REQUIRE(ns == 1, AFEM_EINVAL, "learned preconditioner: training over a base takes one system per sample");
    double om = 0.0;
    AFEM_CUDA(cudaMemcpyAsync(&om, S->omega.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    AFEM_CUDA(cudaStreamSynchronize(st));
    precond_apply_device(c, om, r, S->z64.p);
  }
  forward<double2>(c, S, ns, r, S->z64.p, true, nullptr, nullptr, S->base);
  const int nb = std::min(1024, (int)blocks(n, 256));
  S->part.alloc((size_t)2 * nb * ns);
  S->sums.alloc(2 * ns);
  k_loss_res<<<dim3(nb, ns), 256, 0, st>>>(c->rowptr.p, c->col.p, c->km.p, S->omega.p, n, ns, S->z64.p, r, S->res.p,
                                           S->part.p);
  count_launch();
  k_loss_sum<<<1, 32, 0, st>>>(S->part.p, nb, ns, S->sums.p);
  count_launch();
  k_loss_grad<<<dim3(nb, ns), 256, 0, st>>>(c->rowptr.p, c->col.p, c->km.p, S->omega.p, n, ns, S->res.p, S->sums.p,
                                            S->rms.p, S->s.p, S->dout.p);
  count_launch();
  float* G = S->grad.p;
  k_decode_bwd<<<std::min(1024u, blocks(rows, 256)), 256, 0, st>>>(S->h[L].p, rows, S->dout.p,
                                                                  S->small.p + FIN * H + L * H, S->dh.p,
                                                                  G + off_wout());
  count_launch();
  for (int l = L - 1; l >= 0; --l) {
    k_layer_bwd<<<blocks(rows, ROWS), 128, LAYER_BWD_SMEM, st>>>(rows, S->dh.p, S->sx[l].p, S->sy[l].p,
                                                                 S->wl.p + (size_t)l * XW * H, S->dx.p, G + off_w(l),
                                                                 G + off_c(l));
    count_launch();
    k_agg_bwd<<<dim3(std::min(4096u, blocks(n, 8)), ns), 256, 0, st>>>(c->rowptr.p, c->col.p, c->km.p, S->s.p,
                                                                       S->omega.p, n, S->dx.p, S->dh.p);
    count_launch();
  }
  k_encode_bwd<double2><<<std::min(1024u, blocks(rows, 256)), 256, 0, st>>>(r, n, ns, S->s.p, S->feat.p, S->rms.p,
                                                                            S->dh.p, G + off_win());
  count_launch();
  AFEM_CUDA(cudaGetLastError());
  std::vector<double> h(2 * ns);
  AFEM_CUDA(cudaMemcpyAsync(h.data(), S->sums.p, sizeof(double) * 2 * ns, cudaMemcpyDeviceToHost, st));
  AFEM_CUDA(cudaStreamSynchronize(st));
  double Lsum = 0.0;
  for (int k = 0; k < ns; ++k) Lsum += h[2 * k] / h[2 * k + 1];
  return Lsum;
}

void set_omegas_rms(afem_ctx* c, MpnnState* S, int ns, const double* freq, const double* r_host) {
  std::vector<double> om(ns), rms(ns, 0.0);
  const double pi = 4.0 * std::atan(1.0);
  for (int k = 0; k < ns; ++k) om[k] = 2.0 * pi * freq[k];
  const int n = c->nline;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < ns; ++k) {
      const double re = r_host[2 * ((long)i * ns + k)], im = r_host[2 * ((long)i * ns + k) + 1];
      rms[k] += re * re + im * im;
    }
  for (int k = 0; k < ns; ++k) rms[k] = std::sqrt(rms[k] / n);
  AFEM_CUDA(cudaMemcpyAsync(S->omega.p, om.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, c->stream));
  AFEM_CUDA(cudaMemcpyAsync(S->rms.p, rms.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, c->stream));
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace

void mpnn_destroy(afem_ctx* c) {
  delete c->mpnn;
  c->mpnn = nullptr;
}

int mpnn_nparam() { return NPARAM; }

void mpnn_set_params(afem_ctx* c, const float* p, int np) {
  AFEM_REQUIRE(np == NPARAM, AFEM_EINVAL, "learned preconditioner: wrong number of parameters");
  MpnnState* S = state(c);
  S->p.upload(p, NPARAM, c->stream);
  S->m1.alloc(NPARAM); S->m1.zero(c->stream);
  S->m2.alloc(NPARAM); S->m2.zero(c->stream);
  S->grad.alloc(NPARAM);
  S->adam_t = 0;
  S->cast_valid = false;
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
}

void mpnn_get_params(afem_ctx* c, float* p) {
  MpnnState* S = state(c);
  AFEM_REQUIRE(S->p.p, AFEM_ESTATE, "learned preconditioner: no weights");
  S->p.download(p, NPARAM, c->stream);
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
}

bool mpnn_ready(afem_ctx* c) { return c->mpnn && c->mpnn->p.p; }
int mpnn_base(afem_ctx* c) { return c->mpnn ? c->mpnn->base : 0; }
void mpnn_set_base(afem_ctx* c, int base) {
  AFEM_REQUIRE(base == 0 || base == 1, AFEM_EINVAL, "learned preconditioner: base must be 0 (Jacobi) or 1 (hybrid)");
  state(c)->base = base;
}

// Inside COCG: mpnn_prepare once per solve (omega per system known), then
// mpnn_run per iteration (capturable: kernel launches only; skip = the
// solver's "done" word so a captured chunk past convergence does no work).
void mpnn_prepare(afem_ctx* c, int ns, const double* d_omega) {
  MpnnState* S = state(c);
  ensure_cast(c, S);
  ensure_work(c, S, ns, false);
  AFEM_CUDA(cudaMemcpyAsync(S->omega.p, d_omega, sizeof(double) * ns, cudaMemcpyDeviceToDevice, c->stream));
  rowinfo(c, S, ns);
}

template <class V>
void mpnn_run(afem_ctx* c, int ns, const double* d_rms, const V* r, V* z, const int* skip) {
  MpnnState* S = state(c);
  forward<V>(c, S, ns, r, z, false, d_rms, skip, S->base);
}
template void mpnn_run<double2>(afem_ctx*, int, const double*, const double2*, double2*, const int*);
template void mpnn_run<float2>(afem_ctx*, int, const double*, const float2*, float2*, const int*);

void mpnn_forward_host(afem_ctx* c, int ns, const double* freq, const double* r_host, double* z_host) {
  MpnnState* S = state(c);
  ensure_cast(c, S);
  ensure_work(c, S, ns, false);
  set_omegas_rms(c, S, ns, freq, r_host);
  const long rows = (long)c->nline * ns;
  S->r64.upload(reinterpret_cast<const double2*>(r_host), rows, c->stream);
  S->z64.alloc(rows);
  rowinfo(c, S, ns);
  if (S->base) {
    AFEM_REQUIRE(ns == 1, AFEM_EINVAL, "learned preconditioner: the hybrid base applies to one system at a time");
    precond_apply_device(c, 2.0 * (4.0 * std::atan(1.0)) * freq[0], S->r64.p, S->z64.p);
  }
  forward<double2>(c, S, ns, S->r64.p, S->z64.p, false, nullptr, nullptr, S->base);
  S->z64.download(reinterpret_cast<double2*>(z_host), rows, c->stream);
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
}

// Loss and gradient summed over nsamp residual samples of one frequency (ns = 1 each).
double mpnn_loss_grad_host(afem_ctx* c, double freq, int nsamp, const double* r_host, float* grad_host) {
  MpnnState* S = state(c);
  ensure_cast(c, S);
  ensure_work(c, S, 1, true);
  S->grad.zero(c->stream);
  const int n = c->nline;
  double Lsum = 0.0;
  for (int k = 0; k < nsamp; ++k) {
    set_omegas_rms(c, S, 1, &freq, r_host + 2L * k * n);
    S->r64.upload(reinterpret_cast<const double2*>(r_host + 2L * k * n), n, c->stream);
    Lsum += loss_backward(c, S, 1, S->r64.p);
  }
  if (grad_host) {
    S->grad.download(grad_host, NPARAM, c->stream);
    AFEM_CUDA(cudaStreamSynchronize(c->stream));
  }
  return Lsum;
}

// Adam steps: each step averages the gradient over all nsamp samples.
double mpnn_train_host(afem_ctx* c, double freq, int nsamp, const double* r_host, int steps, float lr,
                       double* hist) {
  MpnnState* S = state(c);
  AFEM_REQUIRE(S->p.p, AFEM_ESTATE, "train: no initial weights");
  const int n = c->nline;
  DBuf<double2> samples;
  samples.upload(reinterpret_cast<const double2*>(r_host), (size_t)nsamp * n, c->stream);
  std::vector<double> rms(nsamp);
  for (int k = 0; k < nsamp; ++k) {
    double a = 0;
    for (int i = 0; i < n; ++i) {
      const double re = r_host[2 * ((long)k * n + i)], im = r_host[2 * ((long)k * n + i) + 1];
      a += re * re + im * im;
    }
    rms[k] = std::sqrt(a / n);
  }
  ensure_work(c, S, 1, true);
  const double om = 2.0 * (4.0 * std::atan(1.0)) * freq;
  AFEM_CUDA(cudaMemcpyAsync(S->omega.p, &om, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  double last = 0.0;
  for (int it = 0; it < steps; ++it) {
    ensure_cast(c, S);
    S->grad.zero(c->stream);
    double Lsum = 0.0;
    for (int k = 0; k < nsamp; ++k) {
      AFEM_CUDA(cudaMemcpyAsync(S->rms.p, &rms[k], sizeof(double), cudaMemcpyHostToDevice, c->stream));
      Lsum += loss_backward(c, S, 1, samples.p + (size_t)k * n);
    }
    S->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - std::pow(b1, (float)S->adam_t), bc2 = 1.f - std::pow(b2, (float)S->adam_t);
    k_adam<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(S->p.p, S->grad.p, S->m1.p, S->m2.p, NPARAM, lr, b1, b2, 1e-8f,
                                                        bc1, bc2, 1.0f / nsamp);
    count_launch();
    S->cast_valid = false;
    last = Lsum / nsamp;
    if (hist) hist[it] = last;
  }
  AFEM_CUDA(cudaStreamSynchronize(c->stream));
  return last;
}

}  // namespace afem
