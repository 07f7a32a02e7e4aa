// learned.cu -- the kernels of the learned initial guess: a small periodic 3D convolutional
// network (U-Net) that maps a voxel image's material fields to the periodic fluctuation of the
// solution of every load case, trained and run by these kernels only.
//
// The reference finds initial guesses by solving the image coarsened by 2 per axis
// (chfem/src/femhmg/femhmg.c:561-846); the network replaces that search, PCG still runs to the
// same tolerance, so results do not change -- only where the iteration starts.
//
// Tensors are FP32, [N][C][D][H][W] with W fastest; every kernel takes the element stride
// between samples (nstride), so a channel slice of a wider tensor (the U-Net's skip
// concatenation) is addressed in place.  Convolutions are periodic (the images are periodic
// cells), 3x3x3 or 1x1x1, cross-correlation: out[co][p] = b[co] + sum_ci sum_o w[co][ci][o]
// in[ci][p + o - 1].
//
// B200 design: direct convolution on the CUDA cores with shared-memory tiles.  A CTA owns a
// 16 (W) x 8 (H) x 4 (D) output tile and 16 output channels; input channels stream through
// shared memory 8 at a time with a 1-voxel periodic halo, the 8 x 27 x 16 weights of the chunk
// next to them; each thread accumulates 4 consecutive W positions x 16 output channels in
// registers, so every shared-memory weight load feeds 4 FMAs and every input load up to 48.
// The weight gradient accumulates per CTA over its tile and adds into the global gradient
// with FP32 atomics (training, unlike the solver, does not need bitwise reproducibility).
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace {

std::string g_err;

constexpr int TX = 16, TY = 8, TZ = 4;      // output tile
constexpr int PT = 4;                        // W positions per thread
constexpr int CO_T = 16;                     // output channels per CTA
constexpr int CI_T = 8;                      // input channels per shared-memory chunk
constexpr int NTH = (TX / PT) * TY * TZ;     // 128 threads
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2, HP = HX * HY * HZ;

__device__ __forceinline__ int pmod(int v, int n) { v %= n; return v < 0 ? v + n : v; }

// Forward convolution (also the backward-data pass, with flipped and transposed weights).
// grid: (tiles of the spatial domain, ceil(Cout / 16), N)
template <int K>
__global__ void __launch_bounds__(NTH) k_conv(const float* __restrict__ in, long in_ns, int Cin, int D, int H, int W,
                                               const float* __restrict__ w, const float* __restrict__ bias, int Cout,
                                               float* __restrict__ out, long out_ns, int relu, int accumulate) {
  constexpr int KK = K * K * K, OFF = K / 2;
  __shared__ float sIn[CI_T * HP];
  __shared__ float sW[CI_T * KK * CO_T];
  const int tilesX = (W + TX - 1) / TX, tilesY = (H + TY - 1) / TY;
  const int tile = blockIdx.x;
  const int x0 = (tile % tilesX) * TX, y0 = ((tile / tilesX) % tilesY) * TY, z0 = (tile / (tilesX * tilesY)) * TZ;
  const int co0 = blockIdx.y * CO_T, n = blockIdx.z;
  const int tid = threadIdx.x;
  const int lx = (tid % (TX / PT)) * PT, ly = (tid / (TX / PT)) % TY, lz = tid / ((TX / PT) * TY);
  const float* inb = in + (long)n * in_ns;
  const long S = (long)D * H * W;
  float acc[CO_T][PT];
#pragma unroll
  for (int c = 0; c < CO_T; c++)
#pragma unroll
    for (int p = 0; p < PT; p++) acc[c][p] = 0.f;
  for (int ci0 = 0; ci0 < Cin; ci0 += CI_T) {
    const int nci = min(CI_T, Cin - ci0);
    __syncthreads();
    // input chunk with periodic halo
    for (int t = tid; t < CI_T * HP; t += NTH) {
      const int c = t / HP, h = t % HP;
      const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
      float v = 0.f;
      if (c < nci) {
        const int gx = pmod(x0 + hx - 1, W), gy = pmod(y0 + hy - 1, H), gz = pmod(z0 + hz - 1, D);
        v = inb[(long)(ci0 + c) * S + ((long)gz * H + gy) * W + gx];
      }
      sIn[t] = v;
    }
    // weights of the chunk: sW[(c * KK + o) * CO_T + co]
    for (int t = tid; t < CI_T * KK * CO_T; t += NTH) {
      const int co = t % CO_T, o = (t / CO_T) % KK, c = t / (CO_T * KK);
      float v = 0.f;
      if (c < nci && co0 + co < Cout) v = w[((long)(co0 + co) * Cin + (ci0 + c)) * KK + o];
      sW[t] = v;
    }
    __syncthreads();
    for (int c = 0; c < nci; c++) {
#pragma unroll
      for (int kz = 0; kz < K; kz++)
#pragma unroll
        for (int ky = 0; ky < K; ky++) {
          // the PT + K - 1 input values of this row
          const float* row = sIn + c * HP + ((lz + kz + 1 - OFF) * HY + (ly + ky + 1 - OFF)) * HX + lx + 1 - OFF;
          float iv[PT + K - 1];
#pragma unroll
          for (int j = 0; j < PT + K - 1; j++) iv[j] = row[j];
#pragma unroll
          for (int kx = 0; kx < K; kx++) {
            const float* wv = sW + (c * KK + (kz * K + ky) * K + kx) * CO_T;
#pragma unroll
            for (int co = 0; co < CO_T; co++) {
              const float wc = wv[co];
#pragma unroll
              for (int p = 0; p < PT; p++) acc[co][p] = fmaf(wc, iv[p + kx], acc[co][p]);
            }
          }
        }
    }
  }
  const int gz = z0 + lz, gy = y0 + ly;
  if (gz >= D || gy >= H) return;
  float* outb = out + (long)n * out_ns;
#pragma unroll
  for (int co = 0; co < CO_T; co++) {
    if (co0 + co >= Cout) break;
    const float b = bias ? bias[co0 + co] : 0.f;
#pragma unroll
    for (int p = 0; p < PT; p++) {
      const int gx = x0 + lx + p;
      if (gx >= W) break;
      const long idx = (long)(co0 + co) * S + ((long)gz * H + gy) * W + gx;
      float v = acc[co][p] + b;
      if (accumulate) v += outb[idx];
      if (relu) v = fmaxf(v, 0.f);
      outb[idx] = v;
    }
  }
}

// Backward-data weights: wt[ci][co][o] = w[co][ci][KK - 1 - o] (flip every axis, swap channels).
__global__ void k_flip_weights(const float* w, int Cout, int Cin, int KK, float* wt) {
  const long n = (long)Cout * Cin * KK;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int o = (int)(t % KK), ci = (int)((t / KK) % Cin), co = (int)(t / ((long)KK * Cin));
    wt[((long)ci * Cout + co) * KK + (KK - 1 - o)] = w[t];
  }
}

// Weight gradient: dw[co][ci][o] += sum_n sum_p g[n][co][p] in[n][ci][p + o - 1]; db[co] += sum g.
// grid: (spatial tiles, ceil(Cout/16) * ceil(Cin/8), N); thread t owns (co, ci) pairs' 27 taps.
template <int K>
__global__ void __launch_bounds__(NTH) k_conv_wgrad(const float* __restrict__ in, long in_ns, int Cin, int D, int H, int W,
                                                     const float* __restrict__ g, long g_ns, int Cout, float* dw, float* db) {
  constexpr int KK = K * K * K, OFF = K / 2;
  extern __shared__ float smem_w[];  // CI_T * HP input values, then CO_T * tile gradients (66 KB)
  float* sIn = smem_w;
  float* sG = smem_w + CI_T * HP;
  const int tilesX = (W + TX - 1) / TX, tilesY = (H + TY - 1) / TY;
  const int tile = blockIdx.x;
  const int x0 = (tile % tilesX) * TX, y0 = ((tile / tilesX) % tilesY) * TY, z0 = (tile / (tilesX * tilesY)) * TZ;
  const int nci_t = (Cin + CI_T - 1) / CI_T;
  const int co0 = (blockIdx.y / nci_t) * CO_T, ci0 = (blockIdx.y % nci_t) * CI_T, n = blockIdx.z;
  const int tid = threadIdx.x;
  const long S = (long)D * H * W;
  const float* inb = in + (long)n * in_ns;
  const float* gb = g + (long)n * g_ns;
  for (int t = tid; t < CI_T * HP; t += NTH) {
    const int c = t / HP, h = t % HP;
    const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
    float v = 0.f;
    if (ci0 + c < Cin) {
      const int gx = pmod(x0 + hx - 1, W), gy = pmod(y0 + hy - 1, H), gz = pmod(z0 + hz - 1, D);
      v = inb[(long)(ci0 + c) * S + ((long)gz * H + gy) * W + gx];
    }
    sIn[t] = v;
  }
  constexpr int TP = TX * TY * TZ;
  for (int t = tid; t < CO_T * TP; t += NTH) {
    const int co = t / TP, p = t % TP;
    const int px = p % TX, py = (p / TX) % TY, pz = p / (TX * TY);
    const int gx = x0 + px, gy = y0 + py, gz = z0 + pz;
    float v = 0.f;
    if (co0 + co < Cout && gx < W && gy < H && gz < D) v = gb[(long)(co0 + co) * S + ((long)gz * H + gy) * W + gx];
    sG[t] = v;
  }
  __syncthreads();
  // thread -> (co, ci) pair; CO_T * CI_T = 128 = NTH
  const int co = tid / CI_T, ci = tid % CI_T;
  if (co0 + co < Cout && ci0 + ci < Cin) {
    float a[KK];
#pragma unroll
    for (int o = 0; o < KK; o++) a[o] = 0.f;
    const float* gp = sG + co * TP;
    const float* ip = sIn + ci * HP;
    for (int p = 0; p < TP; p++) {
      const float gv = gp[p];
      if (gv == 0.f) continue;
      const int px = p % TX, py = (p / TX) % TY, pz = p / (TX * TY);
#pragma unroll
      for (int kz = 0; kz < K; kz++)
#pragma unroll
        for (int ky = 0; ky < K; ky++)
#pragma unroll
          for (int kx = 0; kx < K; kx++)
            a[(kz * K + ky) * K + kx] = fmaf(gv, ip[((pz + kz + 1 - OFF) * HY + (py + ky + 1 - OFF)) * HX + px + kx + 1 - OFF], a[(kz * K + ky) * K + kx]);
    }
#pragma unroll
    for (int o = 0; o < KK; o++) atomicAdd(dw + ((long)(co0 + co) * Cin + (ci0 + ci)) * KK + o, a[o]);
  }
  // bias gradient from the CTAs of the first input-channel chunk
  if (db && ci0 == 0) {
    __syncthreads();
    for (int c = tid; c < CO_T; c += NTH) {
      if (co0 + c >= Cout) continue;
      float s = 0.f;
      for (int p = 0; p < TP; p++) s += sG[c * TP + p];
      atomicAdd(db + co0 + c, s);
    }
  }
}

__global__ void k_relu_bwd(const float* y, long y_ns, float* g, long g_ns, long per_sample, int N) {
  const long tot = per_sample * N;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long n = t / per_sample, i = t % per_sample;
    if (!(y[n * y_ns + i] > 0.f)) g[n * g_ns + i] = 0.f;
  }
}

// 2x2x2 average pool (D, H, W even) and its adjoint (optionally accumulating).
__global__ void k_pool2(const float* in, long in_ns, int C, int D, int H, int W, float* out, long out_ns, int N) {
  const int d = D / 2, h = H / 2, w = W / 2;
  const long per = (long)C * d * h * w, tot = per * N;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long n = t / per, r = t % per;
    const int x = (int)(r % w), y = (int)((r / w) % h), z = (int)((r / ((long)w * h)) % d), c = (int)(r / ((long)w * h * d));
    const float* p = in + n * in_ns + (long)c * D * H * W;
    float s = 0.f;
    for (int dz = 0; dz < 2; dz++)
      for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) s += p[((long)(2 * z + dz) * H + 2 * y + dy) * W + 2 * x + dx];
    out[n * out_ns + r] = 0.125f * s;
  }
}
__global__ void k_pool2_bwd(const float* g, long g_ns, int C, int D, int H, int W, float* gin, long gin_ns, int N, int accumulate) {
  const long per = (long)C * D * H * W, tot = per * N;
  const int d = D / 2, h = H / 2, w = W / 2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long n = t / per, r = t % per;
    const int x = (int)(r % W), y = (int)((r / W) % H), z = (int)((r / ((long)W * H)) % D), c = (int)(r / ((long)W * H * D));
    const float v = 0.125f * g[n * g_ns + (((long)c * d + z / 2) * h + y / 2) * w + x / 2];
    float* o = gin + n * gin_ns + r;
    *o = accumulate ? *o + v : v;
  }
}
// nearest 2x upsample (coarse D, H, W -> 2D, 2H, 2W) and its adjoint
__global__ void k_up2(const float* in, long in_ns, int C, int D, int H, int W, float* out, long out_ns, int N) {
  const int D2 = 2 * D, H2 = 2 * H, W2 = 2 * W;
  const long per = (long)C * D2 * H2 * W2, tot = per * N;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long n = t / per, r = t % per;
    const int x = (int)(r % W2), y = (int)((r / W2) % H2), z = (int)((r / ((long)W2 * H2)) % D2), c = (int)(r / ((long)W2 * H2 * D2));
    out[n * out_ns + r] = in[n * in_ns + (((long)c * D + z / 2) * H + y / 2) * W + x / 2];
  }
}
__global__ void k_up2_bwd(const float* g, long g_ns, int C, int D, int H, int W, float* gin, long gin_ns, int N) {
  const int H2 = 2 * H, W2 = 2 * W;
  const long per = (long)C * D * H * W, tot = per * N;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long n = t / per, r = t % per;
    const int x = (int)(r % W), y = (int)((r / W) % H), z = (int)((r / ((long)W * H)) % D), c = (int)(r / ((long)W * H * D));
    const float* p = g + n * g_ns + (long)c * (2 * D) * H2 * W2;
    float s = 0.f;
    for (int dz = 0; dz < 2; dz++)
      for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) s += p[((long)(2 * z + dz) * H2 + 2 * y + dy) * W2 + 2 * x + dx];
    gin[n * gin_ns + r] = s;
  }
}

// loss = sum (pred - target)^2 / count (FP64 accumulation); grad = 2 (pred - target) / count
__global__ void k_mse(const float* pred, const float* target, long n, double inv_count, float* grad, double* loss) {
  double s = 0.0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const float d = pred[t] - target[t];
    s += (double)d * d;
    if (grad) grad[t] = (float)(2.0 * inv_count) * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_count);
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const float gv = g[t];
    const float mv = b1 * m[t] + (1.f - b1) * gv, vv = b2 * v[t] + (1.f - b2) * gv * gv;
    m[t] = mv;
    v[t] = vv;
    p[t] -= lr * (mv / c1) / (sqrtf(vv / c2) + eps);
  }
}

// Material features of a voxel image: out[n][f][voxel] = table[label][f] (f < F) where the label
// of each voxel is its uint8 colour.
__global__ void k_features(const uint8_t* img, long img_ns, long S, const float* table, int F, float* out, long out_ns, int N) {
  const long tot = S * N;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long n = t / S, i = t % S;
    const int lab = img[n * img_ns + i];
    for (int f = 0; f < F; f++) out[n * out_ns + (long)f * S + i] = table[lab * F + f];
  }
}

// Initial guesses from the network output: x_k[node * 3 + comp] = out[3k + comp][node] plus, on
// the displaced component of load case k, its macroscopic ramp (col for x, (R - row) mod R for y,
// (L - layer) mod L for z; node = row + col R + layer R C).
struct GuessPtrs { double* x[6]; };
__global__ void k_assemble_guess(const float* out, int L, int C, int R, GuessPtrs xs) {
  const long S = (long)L * C * R;
  const int AX[6] = {0, 1, 2, 1, 2, 1}, CO[6] = {0, 1, 2, 2, 0, 0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const double ramp = AX[k] == 0 ? (double)c : (AX[k] == 1 ? (double)((R - r) % R) : (double)((L - l) % L));
#pragma unroll
      for (int comp = 0; comp < 3; comp++)
        xs.x[k][3 * i + comp] = (double)out[(long)(3 * k + comp) * S + i] + (comp == CO[k] ? ramp : 0.0);
    }
  }
}

int grid1(long n) { long g = (n + 255) / 256; return (int)(g < 1 ? 1 : (g > 65535 ? 65535 : g)); }
bool check(const char* who) {
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) { g_err = std::string(who) + ": " + cudaGetErrorString(e); return false; }
  return true;
}
dim3 conv_grid(int N, int D, int H, int W, int Cout) {
  const int tiles = ((W + TX - 1) / TX) * ((H + TY - 1) / TY) * ((D + TZ - 1) / TZ);
  return dim3(tiles, (Cout + CO_T - 1) / CO_T, N);
}

}  // namespace

extern "C" {

const char* chfemB200NnLastError(void) { return g_err.c_str(); }

// out = conv(in) (+ bias) (ReLU when relu) for ksize 3 or 1; accumulate adds into out first.
int chfemB200NnConv3d(const float* in, long in_ns, int N, int Cin, int D, int H, int W, const float* w, const float* bias, int Cout,
                      int ksize, int relu, int accumulate, float* out, long out_ns, void* stream) {
  if (!in || !w || !out || N < 1 || Cin < 1 || Cout < 1 || D < 1 || H < 1 || W < 1 || (ksize != 1 && ksize != 3)) {
    g_err = "chfemB200NnConv3d: bad arguments"; return 0;
  }
  const dim3 g = conv_grid(N, D, H, W, Cout);
  if (ksize == 3) k_conv<3><<<g, NTH, 0, (cudaStream_t)stream>>>(in, in_ns, Cin, D, H, W, w, bias, Cout, out, out_ns, relu, accumulate);
  else k_conv<1><<<g, NTH, 0, (cudaStream_t)stream>>>(in, in_ns, Cin, D, H, W, w, bias, Cout, out, out_ns, relu, accumulate);
  return check("chfemB200NnConv3d") ? 1 : 0;
}

// grad_in = conv^T(grad_out): the forward kernel on flipped, transposed weights (wt: caller
// scratch of Cout*Cin*k^3 floats); accumulate adds into grad_in.
int chfemB200NnConv3dBackwardData(const float* grad_out, long g_ns, int N, int Cout, int D, int H, int W, const float* w, int Cin,
                                  int ksize, float* wt, int accumulate, float* grad_in, long gin_ns, void* stream) {
  if (!grad_out || !w || !wt || !grad_in || (ksize != 1 && ksize != 3)) { g_err = "chfemB200NnConv3dBackwardData: bad arguments"; return 0; }
  const int KK = ksize * ksize * ksize;
  k_flip_weights<<<grid1((long)Cout * Cin * KK), 256, 0, (cudaStream_t)stream>>>(w, Cout, Cin, KK, wt);
  return chfemB200NnConv3d(grad_out, g_ns, N, Cout, D, H, W, wt, nullptr, Cin, ksize, 0, accumulate, grad_in, gin_ns, stream);
}

// dw += dL/dw, db += dL/db (db may be NULL); the caller zeroes them before the first call.
int chfemB200NnConv3dBackwardWeight(const float* in, long in_ns, int N, int Cin, int D, int H, int W, const float* grad_out, long g_ns,
                                    int Cout, int ksize, float* dw, float* db, void* stream) {
  if (!in || !grad_out || !dw || (ksize != 1 && ksize != 3)) { g_err = "chfemB200NnConv3dBackwardWeight: bad arguments"; return 0; }
  const int tiles = ((W + TX - 1) / TX) * ((H + TY - 1) / TY) * ((D + TZ - 1) / TZ);
  const dim3 g(tiles, ((Cout + CO_T - 1) / CO_T) * ((Cin + CI_T - 1) / CI_T), N);
  const size_t smem = (size_t)(CI_T * HP + CO_T * TX * TY * TZ) * sizeof(float);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_conv_wgrad<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_conv_wgrad<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      g_err = "chfemB200NnConv3dBackwardWeight: shared-memory attribute refused"; return 0;
    }
    attr = true;
  }
  if (ksize == 3) k_conv_wgrad<3><<<g, NTH, smem, (cudaStream_t)stream>>>(in, in_ns, Cin, D, H, W, grad_out, g_ns, Cout, dw, db);
  else k_conv_wgrad<1><<<g, NTH, smem, (cudaStream_t)stream>>>(in, in_ns, Cin, D, H, W, grad_out, g_ns, Cout, dw, db);
  return check("chfemB200NnConv3dBackwardWeight") ? 1 : 0;
}

int chfemB200NnReluBackward(const float* y, long y_ns, float* g, long g_ns, long per_sample, int N, void* stream) {
  k_relu_bwd<<<grid1(per_sample * N), 256, 0, (cudaStream_t)stream>>>(y, y_ns, g, g_ns, per_sample, N);
  return check("chfemB200NnReluBackward") ? 1 : 0;
}
int chfemB200NnPool2(const float* in, long in_ns, int N, int C, int D, int H, int W, float* out, long out_ns, void* stream) {
  if ((D | H | W) & 1) { g_err = "chfemB200NnPool2: even sizes only"; return 0; }
  k_pool2<<<grid1((long)C * D * H * W / 8 * N), 256, 0, (cudaStream_t)stream>>>(in, in_ns, C, D, H, W, out, out_ns, N);
  return check("chfemB200NnPool2") ? 1 : 0;
}
int chfemB200NnPool2Backward(const float* g, long g_ns, int N, int C, int D, int H, int W, float* gin, long gin_ns, int accumulate, void* stream) {
  k_pool2_bwd<<<grid1((long)C * D * H * W * N), 256, 0, (cudaStream_t)stream>>>(g, g_ns, C, D, H, W, gin, gin_ns, N, accumulate);
  return check("chfemB200NnPool2Backward") ? 1 : 0;
}
int chfemB200NnUpsample2(const float* in, long in_ns, int N, int C, int D, int H, int W, float* out, long out_ns, void* stream) {
  k_up2<<<grid1((long)C * D * H * W * 8 * N), 256, 0, (cudaStream_t)stream>>>(in, in_ns, C, D, H, W, out, out_ns, N);
  return check("chfemB200NnUpsample2") ? 1 : 0;
}
int chfemB200NnUpsample2Backward(const float* g, long g_ns, int N, int C, int D, int H, int W, float* gin, long gin_ns, void* stream) {
  k_up2_bwd<<<grid1((long)C * D * H * W * N), 256, 0, (cudaStream_t)stream>>>(g, g_ns, C, D, H, W, gin, gin_ns, N);
  return check("chfemB200NnUpsample2Backward") ? 1 : 0;
}
// loss (device double, accumulated) and grad (may be NULL) of the mean squared error
int chfemB200NnMse(const float* pred, const float* target, long n, float* grad, double* loss, void* stream) {
  k_mse<<<grid1(n), 256, 0, (cudaStream_t)stream>>>(pred, target, n, 1.0 / (double)n, grad, loss);
  return check("chfemB200NnMse") ? 1 : 0;
}
int chfemB200NnAdam(float* p, const float* g, float* m, float* v, long n, float lr, float b1, float b2, float eps, int step, void* stream) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid1(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  return check("chfemB200NnAdam") ? 1 : 0;
}
int chfemB200NnFeatures(const uint8_t* img, long img_ns, long S, const float* table, int F, float* out, long out_ns, int N, void* stream) {
  k_features<<<grid1(S * N), 256, 0, (cudaStream_t)stream>>>(img, img_ns, S, table, F, out, out_ns, N);
  return check("chfemB200NnFeatures") ? 1 : 0;
}

// The six elastic initial-guess vectors (device, 3 L C R doubles each) from the network's output
// [18][L][C][R] (device).
int chfemB200NnAssembleGuess(const float* out, int L, int C, int R, double* const* x, void* stream) {
  if (!out || !x) { g_err = "chfemB200NnAssembleGuess: null argument"; return 0; }
  GuessPtrs p;
  for (int k = 0; k < 6; k++) { if (!x[k]) { g_err = "chfemB200NnAssembleGuess: null vector"; return 0; } p.x[k] = x[k]; }
  k_assemble_guess<<<grid1((long)L * C * R), 256, 0, (cudaStream_t)stream>>>(out, L, C, R, p);
  return check("chfemB200NnAssembleGuess") ? 1 : 0;
}

}  // extern "C"
