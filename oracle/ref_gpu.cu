// ref_gpu.cu -- exposes the reference's own GPU kernels through a C ABI.
//
// TEST INFRASTRUCTURE ONLY (the golden-vector generator and GPU parity tests
// load the resulting oracle/_ref/libref_gpu.so; the product never does).
// It compiles the reference translation unit src/rx_host_corr.cu unchanged,
// from where it lies, with a stub DAQIRI header (oracle/stub/daqiri/daqiri.h)
// and its main() renamed, so that k_packAB (:61-72), cgemm_blk_t<ACC>
// (src/cgemm.cuh:28-69), k_diff (:74-77), k_grid_cube (:79-85),
// k_flush_cube (:90-95) and its batched cuFFT plan (:205-206) can be run on
// the same inputs as the X-engine.  Launch shapes follow the reference's own
// call sites (:149, :151, :163, :167-168, :219-222).
#define main ref_main
#include "rx_host_corr.cu"
#undef main

extern "C" {

// Reference build constants (src/rx_host_corr.cu:36-51, src/config.h:26-33).
int ref_const(int which) {
    switch (which) {
        case 0: return MIXER_NANT;
        case 1: return NCUBE;
        case 2: return MIXER_TPKT;
        case 3: return HBATCH;
        case 4: return KPCH;
        case 5: return NG;
        case 6: return NB;
        default: return -1;
    }
}

// k_packAB over one V-update's staged heaps bb[HBATCH][NANT][NB].
int ref_pack(const uint8_t* bb, int8_t* Are, int8_t* Aim, int8_t* Bre, int8_t* Bim, void* st) {
    const int packT = 256;
    const int packG = (int)(((size_t)MIXER_NANT * TOTAL_SAMP + packT - 1) / packT);
    k_packAB<<<packG, packT, 0, (cudaStream_t)st>>>(bb, (MixerI8*)Are, (MixerI8*)Aim, (MixerI8*)Bre,
                                                    (MixerI8*)Bim);
    return (int)cudaGetLastError();
}

// cgemm_blk_t<acc>(M, N, K, ...) over `nbatch` channels, grid as at :149.
int ref_cgemm(int acc, int M, int N, int K, int nbatch, const int8_t* Are, const int8_t* Aim,
              const int8_t* Bre, const int8_t* Bim, int* Cre, int* Cim, void* st) {
    dim3 grid((((M / (MIXER_WT * MIXER_SM)) * (N / (MIXER_WT * MIXER_SN))) * 32 + 255) / 256, 1,
              nbatch);
    if (acc)
        cgemm_blk_t<true><<<grid, 256, 0, (cudaStream_t)st>>>(M, N, K, (const MixerI8*)Are,
                                                                (const MixerI8*)Aim,
                                                                (const MixerI8*)Bre,
                                                                (const MixerI8*)Bim, Cre, Cim);
    else
        cgemm_blk_t<false><<<grid, 256, 0, (cudaStream_t)st>>>(M, N, K, (const MixerI8*)Are,
                                                                 (const MixerI8*)Aim,
                                                                 (const MixerI8*)Bre,
                                                                 (const MixerI8*)Bim, Cre, Cim);
    return (int)cudaGetLastError();
}

// k_flush_cube: Vcube[NCUBE][2][MM][MM] += Vi*, Vi* = 0.
int ref_flush(float* Vcube, int* Vire, int* Viim, void* st) {
    k_flush_cube<<<(unsigned)(((size_t)NCUBE * MN + 255) / 256), 256, 0, (cudaStream_t)st>>>(Vcube, Vire,
                                                                                          Viim);
    return (int)cudaGetLastError();
}

// k_diff over n floats.
int ref_diff(const float* Vs, float* Vp, float* dV, size_t n, void* st) {
    k_diff<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)st>>>(Vs, Vp, dV, n);
    return (int)cudaGetLastError();
}

// cudaMemsetAsync(G) + k_grid_cube (the publish-loop sequence at :220-221).
int ref_grid(const float* dV, float* G, void* st) {
    cudaMemsetAsync(G, 0, (size_t)NCUBE * NG * NG * sizeof(cufftComplex), (cudaStream_t)st);
    k_grid_cube<<<(unsigned)(((size_t)NCUBE * MN + 255) / 256), 256, 0, (cudaStream_t)st>>>(
        dV, (cufftComplex*)G);
    return (int)cudaGetLastError();
}

// The reference's batched plan and forward transform (:205-206, :222).
int ref_fft(const float* G, float* Img, void* st) {
    cufftHandle plan;
    int nfft[2] = {NG, NG};
    if (cufftPlanMany(&plan, 2, nfft, NULL, 1, NG * NG, NULL, 1, NG * NG, CUFFT_C2C, NCUBE) !=
        CUFFT_SUCCESS)
        return -1;
    cufftSetStream(plan, (cudaStream_t)st);
    const cufftResult r =
        cufftExecC2C(plan, (cufftComplex*)G, (cufftComplex*)Img, CUFFT_FORWARD);
    cudaStreamSynchronize((cudaStream_t)st);
    cufftDestroy(plan);
    return r == CUFFT_SUCCESS ? 0 : -2;
}

}  // extern "C"
