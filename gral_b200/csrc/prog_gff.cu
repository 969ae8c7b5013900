// prog_gff.cu -- device pack and unpack of GRAL's flow-field (.gff) and turbulence (.tke) cache
// payloads (GFFWrite.cs, GFFRead.cs).  All kernels are bandwidth-bound streaming passes over one
// situation's full-height fields: 12 bytes of float read and 6 bytes of int16 written per cell
// (TKE: 4 and 2), laid out so that both sides stay coalesced.
#include "prog_gff.cuh"

#include <algorithm>
#include <cmath>

namespace gral {

namespace {

constexpr int kThreads = 256;

// (Int16)(Math.Max(Int16.MinValue, Math.Min(Int16.MaxValue, x * 100))) of GFFWrite.cs:196-216
// and the clamp-then-cast of :296-309, which give the same result for every input: the product
// is clamped to [-32768, 32767] and truncated toward zero; NaN converts to 0 (the x64 JIT's
// truncating conversion of NaN is 0x80000000, whose low 16 bits are 0; newer runtimes saturate
// NaN to 0 as well).  The float-to-int32 conversion saturates and maps NaN to 0, so an integer
// clamp after it gives exactly that.
__device__ __forceinline__ short to_i16_trunc(float x) {
    return (short)max(-32768, min(32767, __float2int_rz(x * 100.0f)));
}

// MathF.Round(x * 100) (round half to even), then the clamp and cast of GFFWrite.cs:446-458.
__device__ __forceinline__ short to_i16_round(float x) {
    return (short)max(-32768, min(32767, __float2int_rn(x * 100.0f)));
}

// (float)(int16 * 0.01F) of GFFRead.cs:223-227, 249-253 and 298-308: one float multiply.
__device__ __forceinline__ float from_i16(short s) { return __fmul_rn((float)s, 0.01f); }

__device__ __forceinline__ size_t col_base(const GffGrid &g, int i, int j) {
    return ((size_t)i * (g.njj + 2) + j) * (g.nkk + 2);
}

// ---- flag -1: i, j outer, k inner, U[k-1], V[k-1], W[k] interleaved (GFFWrite.cs:189-220) ----
// Block 32 x 8: warp y takes one column, its lanes the levels (two passes of 32 levels unrolled,
// so each thread has six loads in flight).  A warp's 32 levels are 128 consecutive bytes of
// each field and 192 consecutive payload bytes; the (i, j) decode happens once per thread.
constexpr int kColsPerBlock = 8;

__global__ void __launch_bounds__(32 * kColsPerBlock) k_pack_columns(GffGrid g, const float *__restrict__ uk,
                                                                     const float *__restrict__ vk,
                                                                     const float *__restrict__ wk,
                                                                     short *__restrict__ out) {
    const int nk = g.nkk + 1, nj = g.njj + 1;
    const unsigned c = blockIdx.x * kColsPerBlock + threadIdx.y;   // payload column (i-1)*nj + (j-1)
    if (c >= (unsigned)(g.nii + 1) * nj) return;
    const int i = c / nj + 1, j = c % nj + 1;
    const float *u = uk + col_base(g, i, j), *v = vk + col_base(g, i, j), *w = wk + col_base(g, i, j) + 1;
    short *o = out + (size_t)c * nk * 3;
    for (int k = threadIdx.x; k < nk; k += 64) {
        const int k2 = k + 32;
        const bool two = k2 < nk;
        const float u0 = u[k], v0 = v[k], w0 = w[k];
        float u1 = 0.f, v1 = 0.f, w1 = 0.f;
        if (two) { u1 = u[k2]; v1 = v[k2]; w1 = w[k2]; }
        o[3 * k] = to_i16_trunc(u0);
        o[3 * k + 1] = to_i16_trunc(v0);
        o[3 * k + 2] = to_i16_trunc(w0);
        if (two) {
            o[3 * k2] = to_i16_trunc(u1);
            o[3 * k2 + 1] = to_i16_trunc(v1);
            o[3 * k2 + 2] = to_i16_trunc(w1);
        }
    }
}

__global__ void __launch_bounds__(32 * kColsPerBlock) k_unpack_columns(GffGrid g, const short *__restrict__ in,
                                                                       float *__restrict__ uk,
                                                                       float *__restrict__ vk,
                                                                       float *__restrict__ wk) {
    const int nk = g.nkk + 1, nj = g.njj + 1;
    const unsigned c = blockIdx.x * kColsPerBlock + threadIdx.y;
    if (c >= (unsigned)(g.nii + 1) * nj) return;
    const int i = c / nj + 1, j = c % nj + 1;
    float *u = uk + col_base(g, i, j), *v = vk + col_base(g, i, j), *w = wk + col_base(g, i, j) + 1;
    const short *p = in + (size_t)c * nk * 3;
    for (int k = threadIdx.x; k < nk; k += 32) {
        const short a = p[3 * k], b = p[3 * k + 1], d = p[3 * k + 2];
        u[k] = from_i16(a);
        v[k] = from_i16(b);
        w[k] = from_i16(d);
    }
}

// ---- flag -2: k outer, rows i, each row U, V, W over j (GFFWrite.cs:277-328) ----
// The fields are k-fastest and the payload j-fastest: a 32x32 (j, k) tile per block goes through
// shared memory, read along k and written along j.  Block 32x8 (32x4 measured slower), grid
// (j tiles, k tiles, rows).
constexpr int kTile = 32, kRowsPerPass = 8;

__global__ void __launch_bounds__(kTile * kRowsPerPass) k_pack_levels(GffGrid g, const float *__restrict__ uk,
                                                                      const float *__restrict__ vk,
                                                                      const float *__restrict__ wk,
                                                                      short *__restrict__ out) {
    __shared__ float tile[3][kTile][kTile + 1];
    const int nj = g.njj + 1, nk = g.nkk + 1, ni = g.nii + 1;
    const int i = blockIdx.z + 1, j0 = blockIdx.x * kTile, k0 = blockIdx.y * kTile;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < kTile; r += kRowsPerPass) {
        const int j = j0 + r + 1, k = k0 + tx + 1;
        if (j <= nj && k <= nk) {
            const size_t b = col_base(g, i, j);
            tile[0][r][tx] = uk[b + k - 1];
            tile[1][r][tx] = vk[b + k - 1];
            tile[2][r][tx] = wk[b + k];
        }
    }
    __syncthreads();
    for (int r = ty; r < kTile; r += kRowsPerPass) {
        const int k = k0 + r + 1, j = j0 + tx + 1;
        if (j <= nj && k <= nk) {
            short *row = out + ((size_t)(k - 1) * ni + (i - 1)) * 3 * nj;
            row[j - 1] = to_i16_trunc(tile[0][tx][r]);
            row[nj + j - 1] = to_i16_trunc(tile[1][tx][r]);
            row[2 * nj + j - 1] = to_i16_trunc(tile[2][tx][r]);
        }
    }
}

__global__ void __launch_bounds__(kTile * kRowsPerPass) k_unpack_levels(GffGrid g, const short *__restrict__ in,
                                                                        float *__restrict__ uk,
                                                                        float *__restrict__ vk,
                                                                        float *__restrict__ wk) {
    __shared__ float tile[3][kTile][kTile + 1];
    const int nj = g.njj + 1, nk = g.nkk + 1, ni = g.nii + 1;
    const int i = blockIdx.z + 1, j0 = blockIdx.x * kTile, k0 = blockIdx.y * kTile;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < kTile; r += kRowsPerPass) {
        const int k = k0 + r + 1, j = j0 + tx + 1;
        if (j <= nj && k <= nk) {
            const short *row = in + ((size_t)(k - 1) * ni + (i - 1)) * 3 * nj;
            tile[0][tx][r] = from_i16(row[j - 1]);
            tile[1][tx][r] = from_i16(row[nj + j - 1]);
            tile[2][tx][r] = from_i16(row[2 * nj + j - 1]);
        }
    }
    __syncthreads();
    for (int r = ty; r < kTile; r += kRowsPerPass) {
        const int j = j0 + r + 1, k = k0 + tx + 1;
        if (j <= nj && k <= nk) {
            const size_t b = col_base(g, i, j);
            uk[b + k - 1] = tile[0][r][tx];
            vk[b + k - 1] = tile[1][r][tx];
            wk[b + k] = tile[2][r][tx];
        }
    }
}

// ---- flag -3: KKART of the inner columns, then per column levels max(KKART,1)..NKK+1 of U, of V,
// of W (GFFWrite.cs:411-499).  One warp per column (i = 1..NII+1, j = 1..NJJ+1); lane 0 of an
// inner column also writes its KKART word. ----
__global__ void __launch_bounds__(kThreads) k_pack_terrain(GffGrid g, const float *__restrict__ uk,
                                                           const float *__restrict__ vk,
                                                           const float *__restrict__ wk,
                                                           const int16_t *__restrict__ kk, int kk_stride,
                                                           const uint32_t *__restrict__ off,
                                                           short *__restrict__ out) {
    const int nj = g.njj + 1;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (long long)(g.nii + 1) * nj) return;
    const int i = (int)(w / nj) + 1, j = (int)(w % nj) + 1;
    const int kkart = kk[((size_t)i * (g.njj + 2) + j) * kk_stride];
    if (lane == 0 && i <= g.nii && j <= g.njj) out[(size_t)(i - 1) * g.njj + (j - 1)] = (short)kkart;
    const int k0 = max(kkart, 1), n = g.nkk + 2 - k0;
    short *o = out + (size_t)g.nii * g.njj + off[w];
    const size_t b = col_base(g, i, j) + k0;
    const float *u = uk + b - 1, *v = vk + b - 1, *wz = wk + b;
    for (int m = lane; m < n; m += 64) {      // two passes of 32 levels with their loads in flight
        const int m2 = m + 32;
        const bool two = m2 < n;
        const float u0 = u[m], v0 = v[m], w0 = wz[m];
        float u1 = 0.f, v1 = 0.f, w1 = 0.f;
        if (two) { u1 = u[m2]; v1 = v[m2]; w1 = wz[m2]; }
        o[m] = to_i16_round(u0);
        o[n + m] = to_i16_round(v0);
        o[2 * n + m] = to_i16_round(w0);
        if (two) {
            o[m2] = to_i16_round(u1);
            o[n + m2] = to_i16_round(v1);
            o[2 * n + m2] = to_i16_round(w1);
        }
    }
}

// GFFRead.cs:274-311: levels below KKART are set to 0 -- the zero-filled output already holds
// that -- the rest from the record.
__global__ void __launch_bounds__(kThreads) k_unpack_terrain(GffGrid g, const short *__restrict__ in,
                                                             const int16_t *__restrict__ kk,
                                                             const uint32_t *__restrict__ off,
                                                             float *__restrict__ uk, float *__restrict__ vk,
                                                             float *__restrict__ wk) {
    const int nj = g.njj + 1;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (long long)(g.nii + 1) * nj) return;
    const int i = (int)(w / nj) + 1, j = (int)(w % nj) + 1;
    const int k0 = max((int)kk[(size_t)i * (g.njj + 2) + j], 1), n = g.nkk + 2 - k0;
    const short *p = in + (size_t)g.nii * g.njj + off[w];
    const size_t b = col_base(g, i, j);
    for (int m = lane; m < n; m += 32) {
        const int k = k0 + m;
        uk[b + k - 1] = from_i16(p[m]);
        vk[b + k - 1] = from_i16(p[n + m]);
        wk[b + k] = from_i16(p[2 * n + m]);
    }
}

// ---- .tke of model 2: TURB of i = 1..NII, j = 1..NJJ, k = 1..NKK (GFFWrite.cs:121-130),
// Convert.ToInt16 of the clamped product: round half to even; NaN makes Convert throw. ----
__global__ void __launch_bounds__(kThreads) k_pack_tke(GffGrid g, const float *__restrict__ turb,
                                                       short *__restrict__ out, int *bad) {
    const long long n = (long long)g.nii * g.njj * g.nkk;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = (int)(t % g.nkk) + 1;
    const long long c = t / g.nkk;
    const int j = (int)(c % g.njj) + 1, i = (int)(c / g.njj) + 1;
    const float x = turb[col_base(g, i, j) + k];
    if (x != x) *bad = 1;
    out[t] = to_i16_round(x);
}

int blocks_for(long long threads) { return (int)((threads + kThreads - 1) / kThreads); }

}  // namespace

long long gff_terrain_offsets(const GffGrid &g, const int16_t *kkart, int stride, std::vector<uint32_t> &off) {
    const int nj = g.njj + 1;
    off.assign((size_t)(g.nii + 1) * nj, 0u);
    long long total = 0;
    size_t w = 0;
    for (int i = 1; i <= g.nii + 1; ++i)
        for (int j = 1; j <= g.njj + 1; ++j, ++w) {
            const int k0 = std::max((int)kkart[((size_t)i * (g.njj + 2) + j) * stride], 1);
            const int n = g.nkk + 2 - k0;
            if (n < 0 || total > 0xffffffffLL) return -1;
            off[w] = (uint32_t)total;
            total += 3LL * n;
        }
    return total;
}

long long gff_data_words(const GffGrid &g, int mode, long long terrain_words) {
    switch (mode) {
        case 0:
        case 1: return 3LL * (g.nii + 1) * (g.njj + 1) * (g.nkk + 1);
        case 2: return (long long)g.nii * g.njj + terrain_words;
        case 3: return (long long)g.nii * g.njj * g.nkk;
        default: return -1;
    }
}

void launch_gff_pack(const GffGrid &g, int mode, const float *uk, const float *vk, const float *wk,
                     const float *turb, const int16_t *kk, int kk_stride, const uint32_t *off, short *out,
                     int *bad, cudaStream_t st) {
    const long long cols = (long long)(g.nii + 1) * (g.njj + 1);
    switch (mode) {
        case 0:
            k_pack_columns<<<(int)((cols + kColsPerBlock - 1) / kColsPerBlock), dim3(32, kColsPerBlock), 0, st>>>(
                g, uk, vk, wk, out);
            break;
        case 1: {
            const dim3 grid((g.njj + 1 + kTile - 1) / kTile, (g.nkk + 1 + kTile - 1) / kTile, g.nii + 1);
            k_pack_levels<<<grid, dim3(kTile, kRowsPerPass), 0, st>>>(g, uk, vk, wk, out);
            break;
        }
        case 2: k_pack_terrain<<<blocks_for(cols * 32), kThreads, 0, st>>>(g, uk, vk, wk, kk, kk_stride, off, out); break;
        case 3: k_pack_tke<<<blocks_for((long long)g.nii * g.njj * g.nkk), kThreads, 0, st>>>(g, turb, out, bad); break;
        default: break;
    }
}

void launch_gff_unpack(const GffGrid &g, int flag, const short *in, const int16_t *kk, const uint32_t *off,
                       float *uk, float *vk, float *wk, cudaStream_t st) {
    const long long cols = (long long)(g.nii + 1) * (g.njj + 1);
    if (flag == -1) {
        k_unpack_columns<<<(int)((cols + kColsPerBlock - 1) / kColsPerBlock), dim3(32, kColsPerBlock), 0, st>>>(
            g, in, uk, vk, wk);
    } else if (flag == -2) {
        const dim3 grid((g.njj + 1 + kTile - 1) / kTile, (g.nkk + 1 + kTile - 1) / kTile, g.nii + 1);
        k_unpack_levels<<<grid, dim3(kTile, kRowsPerPass), 0, st>>>(g, in, uk, vk, wk);
    } else if (flag == -3) {
        k_unpack_terrain<<<blocks_for(cols * 32), kThreads, 0, st>>>(g, in, kk, off, uk, vk, wk);
    }
}

}  // namespace gral
