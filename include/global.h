/* Drop-in replacement for the reference's cudasymmfft/global.h: the transform
 * kind enum with the same enumerators and values (global.h:6-15), which are
 * part of the do_transform ABI, and the TRANS_BLOCK_DIM macro (global.h:5) for
 * callers that size their own blocks with it.  The reference's cuFFT
 * error-string table is not needed: no cuFFT is used. */
#ifndef __GLOBAL__
#define __GLOBAL__

#define TRANS_BLOCK_DIM 16

enum transform_kind {
    DCT_1,
    DCT_2,
    DCT_3,
    DST_1,
    DST_2,
    DST_3,
    DFT_R2C,
    DFT_C2R
};

#endif /* __GLOBAL__ */
