// prog_gff.cuh -- GRAL flow-field (.gff) and turbulence (.tke) cache payloads on the device:
// packing the solved fields into the int16 formats of GFFWrite.cs and reading them back
// (GFFRead.cs).  The zip container around the payload stays with the host.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace gral {

struct GffGrid {
    int nii, njj, nkk;   // fields are flat [nii+2][njj+2][nkk+2], k fastest
};

// Terrain format (flag -3): offset in int16 words of each column's record (i = 1..nii+1 outer,
// j = 1..njj+1 inner) from the start of the records, which follow the nii*njj KKART words.  A
// record holds 3*(nkk+2-max(KKART,1)) words.  Returns the total words of all records, or -1 when
// a KKART above nkk+2 leaves a negative record length (GFFWrite.cs:438 and GFFRead.cs:283 fail).
// kkart: flat [nii+2][njj+2] with `stride` int16 words between columns.
long long gff_terrain_offsets(const GffGrid &g, const int16_t *kkart, int stride, std::vector<uint32_t> &off);

// Payload words after the 32-byte header (modes as GRAL_GFF_* in gral_prog.h); terrain_words is
// the total of gff_terrain_offsets.
long long gff_data_words(const GffGrid &g, int mode, long long terrain_words);

// Packs one situation's fields into `out` (device, gff_data_words int16 words).  Mode 2 needs the
// device KKART (`kk`, `kk_stride` words between columns) and record offsets; mode 3 reads `turb`
// and sets *bad (device) to 1 on a non-finite value.
void launch_gff_pack(const GffGrid &g, int mode, const float *uk, const float *vk, const float *wk,
                     const float *turb, const int16_t *kk, int kk_stride, const uint32_t *off, short *out,
                     int *bad, cudaStream_t st);

// Reads payload words `in` (device, after the header) of flag -1, -2 or -3 into zero-filled flat
// fields uk, vk, wk (device).  Flag -3 needs the device KKART (flat, stride 1) and record offsets.
void launch_gff_unpack(const GffGrid &g, int flag, const short *in, const int16_t *kk, const uint32_t *off,
                       float *uk, float *vk, float *wk, cudaStream_t st);

}  // namespace gral
