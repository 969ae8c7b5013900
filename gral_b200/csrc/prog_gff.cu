// prog_gff.cu -- device pack and unpack of GRAL's flow-field (.gff) and turbulence (.tke) cache
// payloads (GFFWrite.cs, GFFRead.cs).  All kernels are bandwidth-bound streaming passes over one
// situation's full-height fields: 12 bytes of float read and 6 bytes of int16 written per cell
// (TKE: 4 and 2), laid out so that both sides stay coalesced.
#include "prog_gff.cuh"

#include <cstdlib>
#include <cstring>

#include "prog_ctx.cuh"

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

// ---- C ABI: gral_prog_gff_* (include/gral_prog.h) ----

using namespace gral;

namespace {

void put_header(uint8_t *out, int32_t nkk, int32_t njj, int32_t nii, float dir, float speed, int32_t stab,
                float dxk, int32_t flag) {
    const int32_t a[3] = {nkk, njj, nii};
    std::memcpy(out, a, 12);
    std::memcpy(out + 12, &dir, 4);
    std::memcpy(out + 16, &speed, 4);
    std::memcpy(out + 20, &stab, 4);
    std::memcpy(out + 24, &dxk, 4);
    std::memcpy(out + 28, &flag, 4);
}

int *gff_bad_flag(gral_ctx *ctx, long long words) {
    return reinterpret_cast<int *>(ctx->gff.p + words + (words & 1));
}

int gff_words(gral_ctx *ctx, int mode, long long *words, std::vector<uint32_t> *off) {
    const GffGrid g{ctx->nii, ctx->njj, ctx->nkk};
    long long terrain = 0;
    if (mode == GRAL_GFF_TERRAIN) {
        std::vector<uint32_t> tmp;
        terrain = gff_terrain_offsets(g, ctx->h_kkart.data(), 1, off ? *off : tmp);
        if (terrain < 0) return fail(ctx, GRAL_EINVAL, "KKART above NKK+1 leaves no room for a terrain-format record");
    }
    *words = gff_data_words(g, mode, terrain);
    return GRAL_OK;
}

}  // namespace

extern "C" {

int gral_prog_gff_size(gral_ctx *ctx, int32_t mode, uint64_t *bytes) {
    if (!ctx || !bytes) return GRAL_EINVAL;
    if (mode < GRAL_GFF_COLUMNS || mode > GRAL_GFF_TKE) return fail(ctx, GRAL_EINVAL, "unknown payload mode");
    if (!ctx->loaded) return fail(ctx, GRAL_ESTATE, "payload size before load");
    long long words = 0;
    const int rc = gff_words(ctx, mode, &words, nullptr);
    if (rc != GRAL_OK) return rc;
    *bytes = GRAL_GFF_HEADER_BYTES + 2 * (uint64_t)words;
    return GRAL_OK;
}

}  // extern "C"

namespace {

// Checks a pack request and prepares its device buffers (payload words, terrain offsets, the
// cleared TKE error flag); *words receives the payload words after the header.
int gff_pack_prepare(gral_ctx *ctx, int32_t situation, int32_t mode, long long *words) {
    if (mode < GRAL_GFF_COLUMNS || mode > GRAL_GFF_TKE) return fail(ctx, GRAL_EINVAL, "unknown payload mode");
    if (!ctx->loaded || !ctx->stored) return fail(ctx, GRAL_ESTATE, "payload pack before store");
    if (situation < 0 || situation >= ctx->nb) return fail(ctx, GRAL_EINVAL, "situation index out of range");
    if (mode == GRAL_GFF_TKE && ctx->model != 2)
        return fail(ctx, GRAL_EINVAL, "the turbulence payload needs turbulence model 2");
    if (mode == GRAL_GFF_LEVELS && ctx->nii + 1 > 65535) return fail(ctx, GRAL_ETOOLARGE, "more than 65534 rows");
    CK(cudaSetDevice(ctx->device));
    std::vector<uint32_t> off;
    int rc = gff_words(ctx, mode, words, &off);
    if (rc != GRAL_OK) return rc;
    cudaStream_t st = ctx->stream;
    CK(ctx->gff.ensure((size_t)*words + 3));   // spare words: the mode-3 error flag, 4-byte aligned
    if (mode == GRAL_GFF_TERRAIN) {
        CK(ctx->gffoff.ensure(off.size()));
        CK(cudaMemcpyAsync(ctx->gffoff.p, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    }
    if (mode == GRAL_GFF_TKE) CK(cudaMemsetAsync(gff_bad_flag(ctx, *words), 0, sizeof(int), st));
    return GRAL_OK;
}

void gff_pack_launch(gral_ctx *ctx, int32_t situation, int32_t mode, long long words) {
    const GffGrid g{ctx->nii, ctx->njj, ctx->nkk};
    const size_t o = ctx->sg.stride * (size_t)situation;
    launch_gff_pack(g, mode, ctx->sg.uk + o, ctx->sg.vk + o, ctx->sg.wk + o,
                    ctx->model == 2 ? ctx->sg.turb + o : nullptr,
                    reinterpret_cast<const int16_t *>(ctx->meta.p), (int)(sizeof(ColMeta) / sizeof(int16_t)),
                    ctx->gffoff.p, ctx->gff.p, gff_bad_flag(ctx, words), ctx->stream);
}

}  // namespace

extern "C" {

int gral_prog_gff_pack(gral_ctx *ctx, int32_t situation, int32_t mode, float wind_dir, float wind_speed,
                       int32_t stability_class, uint8_t *out, uint64_t capacity) {
    if (!ctx) return GRAL_EINVAL;
    if (!out) return fail(ctx, GRAL_EINVAL, "null output buffer");
    long long words = 0;
    int rc = gff_pack_prepare(ctx, situation, mode, &words);
    if (rc != GRAL_OK) return rc;
    if (capacity < GRAL_GFF_HEADER_BYTES + 2 * (uint64_t)words)
        return fail(ctx, GRAL_EINVAL, "output buffer smaller than the payload");
    cudaStream_t st = ctx->stream;
    int *bad = gff_bad_flag(ctx, words);
    gff_pack_launch(ctx, situation, mode, words);
    CK(cudaGetLastError());
    int hbad = 0;
    if (mode == GRAL_GFF_TKE) CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out + GRAL_GFF_HEADER_BYTES, ctx->gff.p, 2 * (size_t)words, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hbad) return fail(ctx, GRAL_ENONFINITE, "non-finite TKE value: the reference's conversion fails there");
    const int32_t nkk_word = (mode == GRAL_GFF_LEVELS || mode == GRAL_GFF_TERRAIN) ? -ctx->nkk : ctx->nkk;
    const int32_t flag = (mode == GRAL_GFF_TKE) ? -1 : -1 - mode;
    put_header(out, nkk_word, ctx->njj, ctx->nii, wind_dir, wind_speed, stability_class, ctx->params[0].dxk, flag);
    return GRAL_OK;
}

int gral_prog_gff_pack_timed(gral_ctx *ctx, int32_t situation, int32_t mode, int32_t repeats, double *kernel_ms) {
    if (!ctx) return GRAL_EINVAL;
    if (repeats < 1 || !kernel_ms) return fail(ctx, GRAL_EINVAL, "repeats must be positive and kernel_ms set");
    long long words = 0;
    int rc = gff_pack_prepare(ctx, situation, mode, &words);
    if (rc != GRAL_OK) return rc;
    cudaStream_t st = ctx->stream;
    const size_t flush = 256u << 20;
    CK(ctx->l2flush.ensure(flush));
    double sum = 0.0;
    for (int r = 0; r < repeats; ++r) {
        CK(cudaMemsetAsync(ctx->l2flush.p, r & 0xff, flush, st));
        CK(cudaEventRecord(ctx->ev[0], st));
        gff_pack_launch(ctx, situation, mode, words);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ctx->ev[1], st));
        CK(cudaEventSynchronize(ctx->ev[1]));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        sum += ms;
    }
    *kernel_ms = sum / repeats;
    return GRAL_OK;
}

int gral_prog_gff_unpack(gral_ctx *ctx, const uint8_t *payload, uint64_t bytes, int32_t nii, int32_t njj,
                         int32_t nkk, float dxk, const int16_t *kkart, float *uk, float *vk, float *wk,
                         float *wind_dir, float *wind_speed, int32_t *stability_class, int32_t *format) {
    if (!ctx) return GRAL_EINVAL;
    if (!payload || !uk || !vk || !wk) return fail(ctx, GRAL_EINVAL, "null pointer");
    if (nii < 1 || njj < 1 || nkk < 1) return fail(ctx, GRAL_EINVAL, "bad grid dimensions");
    if (nii > ctx->cap_nii || njj > ctx->cap_njj || nkk > ctx->cap_nkk)
        return fail(ctx, GRAL_EINVAL, "grid exceeds the context's capacity");
    if (bytes < GRAL_GFF_HEADER_BYTES) return fail(ctx, GRAL_EINVAL, "payload shorter than its header");
    int32_t h[8];
    std::memcpy(h, payload, sizeof(h));
    float dir, speed, cell;
    std::memcpy(&dir, payload + 12, 4);
    std::memcpy(&speed, payload + 16, 4);
    std::memcpy(&cell, payload + 24, 4);
    // GFFRead.cs:185-208: Math.Abs of the first word (which throws for int.MinValue), then the
    // grid and the cell size must equal the model's
    if (h[0] == INT32_MIN || std::abs(h[0]) != nkk)
        return fail(ctx, GRAL_EINVAL, "field dimension in z-direction does not match");
    if (h[1] != njj) return fail(ctx, GRAL_EINVAL, "field dimension in y-direction does not match");
    if (h[2] != nii) return fail(ctx, GRAL_EINVAL, "field dimension in x-direction does not match");
    if (cell != dxk) return fail(ctx, GRAL_EINVAL, "horizontal grid size does not match");
    const int32_t flag = h[7];
    if (wind_dir) *wind_dir = dir;
    if (wind_speed) *wind_speed = speed;
    if (stability_class) *stability_class = h[5];
    if (format) *format = flag;
    if (flag != -1 && flag != -2 && flag != -3) return GRAL_OK;   // the reference reads nothing more
    if (flag == -2 && nii + 1 > 65535) return fail(ctx, GRAL_ETOOLARGE, "more than 65534 rows");
    const GffGrid g{nii, njj, nkk};
    const size_t ncols = (size_t)(nii + 2) * (njj + 2), cells = ncols * (nkk + 2);
    std::vector<uint32_t> off;
    long long words;
    if (flag == -3) {
        if (!kkart) return fail(ctx, GRAL_EINVAL, "the terrain format needs the domain's KKART");
        const long long terrain = gff_terrain_offsets(g, kkart, 1, off);
        if (terrain < 0) return fail(ctx, GRAL_EINVAL, "KKART above NKK+1 leaves no room for a terrain-format record");
        words = gff_data_words(g, 2, terrain);
        if (bytes - GRAL_GFF_HEADER_BYTES < 2 * (uint64_t)words)
            return fail(ctx, GRAL_EINVAL, "payload shorter than its grid");
        // GFFRead.cs:260-272: the file's KKART must be the model's
        const uint8_t *kb = payload + GRAL_GFF_HEADER_BYTES;
        for (int i = 1; i <= nii; ++i)
            for (int j = 1; j <= njj; ++j) {
                int16_t v;
                std::memcpy(&v, kb + 2 * ((size_t)(i - 1) * njj + (j - 1)), 2);
                if (v != kkart[(size_t)i * (njj + 2) + j])
                    return fail(ctx, GRAL_EINVAL, "building or terrain of flow field does not match");
            }
    } else {
        words = gff_data_words(g, 0, 0);
        if (bytes - GRAL_GFF_HEADER_BYTES < 2 * (uint64_t)words)
            return fail(ctx, GRAL_EINVAL, "payload shorter than its grid");
    }
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    CK(ctx->gff.ensure((size_t)words + 2));
    CK(ctx->gffu.ensure(3 * cells));
    CK(cudaMemcpyAsync(ctx->gff.p, payload + GRAL_GFF_HEADER_BYTES, 2 * (size_t)words, cudaMemcpyHostToDevice, st));
    if (flag == -3) {
        CK(ctx->gffoff.ensure(off.size()));
        CK(ctx->gffkk.ensure(ncols));
        CK(cudaMemcpyAsync(ctx->gffoff.p, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->gffkk.p, kkart, ncols * sizeof(int16_t), cudaMemcpyHostToDevice, st));
    }
    float *du = ctx->gffu.p, *dv = du + cells, *dw = dv + cells;
    CK(cudaMemsetAsync(du, 0, 3 * cells * sizeof(float), st));
    launch_gff_unpack(g, flag, ctx->gff.p, ctx->gffkk.p, ctx->gffoff.p, du, dv, dw, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(uk, du, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(vk, dv, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(wk, dw, cells * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return GRAL_OK;
}

}  // extern "C"
