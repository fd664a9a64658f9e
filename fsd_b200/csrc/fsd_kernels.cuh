// Host-side launchers of the device kernels (one translation unit each).
#pragma once

#include "fsd_internal.h"

namespace fsd {

// nlist.cu
size_t scan_scratch_elems(int n);
void exclusive_scan(const unsigned* in, unsigned* out, int n, unsigned* scratch, cudaStream_t st);
void counting_sort(const unsigned* key, int n, int nbins, unsigned* count, unsigned* start, unsigned* fill,
                   unsigned* items, unsigned* scan_scratch, cudaStream_t st);
int3 cell_dims(const Box& b, float rlist);
int build_neighbor_list(fsd_handle* h, const float4* pos, int* max_count_host);
int build_lub_list(fsd_handle* h, const float4* pos);
int init_particle_order(fsd_handle* h);

// mobility.cu
struct FFTPlan {
    int n;
    int nst;
    int radix[12];
};
FFTPlan make_fft_plan(int n);
void fill_twiddles(fsd_handle* h);
int mobility_bin_particles(fsd_handle* h, const float4* pos);
void mobility_set_gridk(fsd_handle* h);
// genU (11N) = M genF (11N); parts: 1 wave, 2 real+self, 3 both.  When
// saddle_x is non-null, genU[0:6N] += saddle_x[11N:17N] (Saddle.cu:118-124).
int mobility_apply(fsd_handle* h, const float4* pos, const float* genF, float* genU, int parts,
                   const float* saddle_x, bool rebin);
// Wave-space part driven by a grid already holding spectra (Brownian):
// inverse FFT + contraction into w.uwave.
void mobility_wave_from_spectrum(fsd_handle* h, const float4* pos);
void mobility_combine(fsd_handle* h, const float4* pos, const float* genF, float* genU, bool wave, bool real,
                      const float* saddle_x);

// lubrication.cu
void lub_rfu(fsd_handle* h, const float4* pos, const float* U, float* F, const float* saddle_x);
void lub_rfe(fsd_handle* h, const float4* pos, float shear_rate, const float3* ori, const float* b2mask, float B2,
             float* F);
void lub_rsu(fsd_handle* h, const float4* pos, const float* U, float* S);
void lub_rse(fsd_handle* h, const float4* pos, float shear_rate, const float3* ori, const float* b2mask, float B2,
             float* S);

}  // namespace fsd
