// Compiled size-specialized tile kernels:
//   X(shard, N, P, T, OP, MODE, SIGN, TW4, STAGES, MINB, TWB, radices...)
// MINB is the CTAs-per-SM register target (__launch_bounds__), chosen so
// that the kernel does not spill.  TWB holds the sk_kernel.cuh SK_* bits:
// 1 basis (else full) pass twiddles, 2 twiddles staged in shared memory,
// 4 mirrored butterfly pairs in the real tiles' last (R2C) or first (C2R)
// pass, 8 pass 0 from the staging buffer into a separate work buffer.
// Every other length runs on the generic tile kernel.  The shard index
// spreads the instantiations over parallel compile units.  Several entries
// for the same (N, OP, MODE, SIGN, TW4) are variants of the tile shape or
// register target: the first is the planner's default, the others are
// selected by the sk-variant planner hint (and timed by the autotuner).
#pragma once

#define SIP_SK_CONFIGS(X)                                                     \
    /* 1D / last-axis C2C rows (split pass 0, TWB 9) */                       \
    X(0, 4096, 1, 128, OP_C2C, SK_ROWS, -1, false, 2, 3, 9, 16, 16, 16)              \
    X(1, 4096, 1, 128, OP_C2C, SK_ROWS, 1, false, 2, 3, 9, 16, 16, 16)               \
    X(2, 2048, 1, 128, OP_C2C, SK_ROWS, -1, false, 2, 4, 9, 16, 16, 8)               \
    X(3, 2048, 1, 128, OP_C2C, SK_ROWS, 1, false, 2, 4, 9, 16, 16, 8)                \
    X(4, 1024, 4, 256, OP_C2C, SK_ROWS, -1, false, 2, 2, 9, 16, 16, 4)               \
    X(5, 1024, 4, 256, OP_C2C, SK_ROWS, 1, false, 2, 2, 9, 16, 16, 4)                \
    /* rows of 256: 16 per 128-thread CTA with staged twiddles (the last    \
       axis of 256^3: 43.7 us against 48.5 with 8 per CTA, the variant) */   \
    X(6, 256, 16, 128, OP_C2C, SK_ROWS, -1, false, 2, 3, 11, 16, 16)                 \
    X(7, 256, 16, 128, OP_C2C, SK_ROWS, 1, false, 2, 3, 11, 16, 16)                  \
    X(6, 256, 8, 128, OP_C2C, SK_ROWS, -1, false, 2, 4, 9, 16, 16)                   \
    X(7, 256, 8, 128, OP_C2C, SK_ROWS, 1, false, 2, 4, 9, 16, 16)                    \
    X(0, 8192, 1, 256, OP_C2C, SK_ROWS, -1, false, 2, 1, 9, 32, 16, 16)              \
    X(1, 8192, 1, 256, OP_C2C, SK_ROWS, 1, false, 2, 1, 9, 32, 16, 16)               \
    /* strided axes of 2D / 3D transforms */                                  \
    /* 2048-point columns: radix 32 first, 256 threads (200 us against 212 \
       for 2048^2 x 8 with 16, 16, 8 on 512 threads, the hint variant) */    \
    X(2, 2048, 8, 256, OP_C2C, SK_COLS, -1, false, 1, 1, 1, 32, 8, 8)                \
    X(3, 2048, 8, 256, OP_C2C, SK_COLS, 1, false, 1, 1, 1, 32, 8, 8)                 \
    X(2, 2048, 8, 512, OP_C2C, SK_COLS, -1, false, 1, 1, 1, 16, 16, 8)               \
    X(3, 2048, 8, 512, OP_C2C, SK_COLS, 1, false, 1, 1, 1, 16, 16, 8)                \
    /* 256-point column and transposed-row passes: 16 transforms per       \
       128-thread CTA with a split pass 0, twiddles staged in the column   \
       pass (C2C 65536 x 4096: 1.69 ms against 1.84 with 256-thread CTAs);   \
       the 256-thread form is a hint variant */                              \
    X(4, 256, 16, 128, OP_C2C, SK_COLS, -1, false, 2, 3, 11, 16, 16)                 \
    X(5, 256, 16, 128, OP_C2C, SK_COLS, 1, false, 2, 3, 11, 16, 16)                  \
    X(6, 256, 16, 128, OP_C2C, SK_COLS, -1, true, 2, 3, 11, 16, 16)                  \
    X(7, 256, 16, 128, OP_C2C, SK_COLS, 1, true, 2, 3, 11, 16, 16)                   \
    X(0, 256, 16, 128, OP_C2C, SK_ROWS_T, -1, false, 2, 3, 9, 16, 16)                \
    X(1, 256, 16, 128, OP_C2C, SK_ROWS_T, 1, false, 2, 3, 9, 16, 16)                 \
    X(4, 256, 16, 256, OP_C2C, SK_COLS, -1, false, 2, 3, 1, 16, 16)                  \
    X(5, 256, 16, 256, OP_C2C, SK_COLS, 1, false, 2, 3, 1, 16, 16)                   \
    /* four-step 65536 = 256 x 256 */                                         \
    X(6, 256, 16, 256, OP_C2C, SK_COLS, -1, true, 2, 3, 1, 16, 16)                   \
    X(7, 256, 16, 256, OP_C2C, SK_COLS, 1, true, 2, 3, 1, 16, 16)                    \
    X(0, 256, 16, 256, OP_C2C, SK_ROWS_T, -1, false, 2, 3, 1, 16, 16)                \
    X(1, 256, 16, 256, OP_C2C, SK_ROWS_T, 1, false, 2, 3, 1, 16, 16)                 \
    /* four-step 2^19 = 512 x 1024 (real 2^20) */                             \
    /* 8 columns per 128-thread CTA, staged twiddles, split pass 0 (C2R    \
       2^20 x 256 pass A: 585 us against 602 with 16 per 256-thread CTA) */  \
    X(2, 512, 8, 128, OP_C2C, SK_COLS, -1, true, 2, 3, 11, 16, 32)                   \
    X(2, 512, 16, 256, OP_C2C, SK_COLS, -1, true, 1, 3, 1, 16, 32)                   \
    X(3, 512, 8, 128, OP_C2C, SK_COLS, 1, true, 2, 3, 11, 16, 32)                    \
    X(3, 512, 16, 256, OP_C2C, SK_COLS, 1, true, 1, 3, 1, 16, 32)                    \
    /* pass B on rows of 1024: staged twiddles, split pass 0, double       \
       buffer (C2R 2^20 x 256: 409 us against 435 single-buffered) */        \
    X(4, 1024, 8, 256, OP_C2C, SK_ROWS_T, -1, false, 2, 1, 11, 32, 32)               \
    X(5, 1024, 8, 256, OP_C2C, SK_ROWS_T, 1, false, 2, 1, 11, 32, 32)                \
    X(4, 1024, 8, 256, OP_C2C, SK_ROWS_T, -1, false, 1, 3, 1, 32, 32)                \
    X(5, 1024, 8, 256, OP_C2C, SK_ROWS_T, 1, false, 1, 3, 1, 32, 32)                 \
    /* real rows: R2C / C2R of N = 1000, 6000 (half length 500, 3000).  The  \
       defaults split pass 0 (TWB 8: staging buffer -> work buffer, next tile \
       staged after it), keep the twiddles in shared memory (2) and, for     \
       R2C, run the last pass as mirrored butterfly pairs with the post-     \
       process fused (4); small CTAs (2-4 warps) leave more of them per SM.  \
       The second entry of a length is a hint variant. */                    \
    X(0, 500, 2, 64, OP_R2C_HALF, SK_ROWS, -1, false, 2, 8, 15, 25, 5, 4)            \
    X(1, 500, 4, 128, OP_C2R_HALF, SK_ROWS, 1, false, 2, 4, 11, 20, 25)              \
    X(2, 3000, 1, 128, OP_R2C_HALF, SK_ROWS, -1, false, 2, 4, 15, 25, 15, 8)         \
    X(3, 3000, 2, 256, OP_C2R_HALF, SK_ROWS, 1, false, 2, 2, 11, 25, 8, 15)          \
    X(7, 3000, 1, 128, OP_C2R_HALF, SK_ROWS, 1, false, 2, 4, 9, 25, 8, 15)           \
    X(4, 3000, 1, 128, OP_R2C_HALF, SK_ROWS, -1, false, 2, 4, 7, 15, 25, 8)          \
    X(5, 3000, 2, 256, OP_C2R_HALF, SK_ROWS, 1, false, 2, 2, 1, 25, 8, 15)           \
    /* real rows of N = 2048, 4096, 8192 (half lengths 1024, 2048, 4096) */  \
    X(6, 1024, 4, 256, OP_R2C_HALF, SK_ROWS, -1, false, 2, 2, 15, 16, 16, 4)         \
    X(7, 1024, 4, 256, OP_C2R_HALF, SK_ROWS, 1, false, 2, 2, 11, 16, 16, 4)          \
    X(0, 2048, 1, 128, OP_R2C_HALF, SK_ROWS, -1, false, 2, 4, 15, 16, 16, 8)         \
    X(1, 2048, 1, 128, OP_C2R_HALF, SK_ROWS, 1, false, 2, 4, 15, 8, 16, 16)          \
    X(2, 4096, 1, 256, OP_R2C_HALF, SK_ROWS, -1, false, 2, 2, 15, 16, 32, 8)         \
    X(3, 4096, 1, 256, OP_C2R_HALF, SK_ROWS, 1, false, 2, 2, 15, 16, 16, 16)         \
    X(4, 1024, 4, 256, OP_R2C_HALF, SK_ROWS, -1, false, 2, 3, 7, 16, 16, 4)          \
    X(5, 2048, 1, 128, OP_R2C_HALF, SK_ROWS, -1, false, 2, 4, 7, 16, 16, 8)          \
    X(6, 4096, 1, 256, OP_R2C_HALF, SK_ROWS, -1, false, 2, 2, 7, 16, 32, 8)          \
    /* 2D 500 x 50 (the reference's MRI example shape): rows of 50, columns \
       of 500 over the 50-wide slices */                                     \
    X(2, 50, 16, 128, OP_C2C, SK_ROWS, -1, false, 2, 4, 1, 5, 10)                    \
    X(3, 50, 16, 128, OP_C2C, SK_ROWS, 1, false, 2, 4, 1, 5, 10)                     \
    X(4, 500, 10, 256, OP_C2C, SK_COLS, -1, false, 2, 2, 1, 25, 20)                  \
    X(5, 500, 10, 256, OP_C2C, SK_COLS, 1, false, 2, 2, 1, 25, 20)                   \
    /* odd real length 2187 = 3^7, two rows per complex FFT (the R2C tile  \
       shape from a run-time compiled sweep: 4 % faster than 2 x 192) */     \
    X(7, 2187, 2, 128, OP_R2C_PAIR, SK_ROWS, -1, false, 2, 3, 15, 27, 9, 9)          \
    /* C2R: one row pair per 128-thread CTA, four CTAs per SM (542 us for  \
       122741 rows against 573 us with two pairs per 192-thread CTA) */      \
    X(4, 2187, 1, 128, OP_C2R_PAIR, SK_ROWS, 1, false, 2, 4, 11, 27, 9, 9)           \
    X(0, 2187, 2, 192, OP_C2R_PAIR, SK_ROWS, 1, false, 2, 2, 11, 27, 9, 9)           \
    X(3, 2187, 2, 192, OP_C2R_PAIR, SK_ROWS, 1, false, 2, 2, 9, 27, 9, 9)            \
    X(1, 2187, 2, 128, OP_R2C_PAIR, SK_ROWS, -1, false, 2, 3, 1, 27, 9, 9)           \
    X(2, 2187, 2, 192, OP_C2R_PAIR, SK_ROWS, 1, false, 2, 2, 1, 27, 9, 9)            \
    /* real 2^20 fused four-step: R2C pass B + post, C2R pre + pass A        \
       (planner hint) */                                                     \
    X(4, 1024, 16, 512, OP_R2C_4B, SK_ROWS_T, -1, false, 1, 1, 1, 32, 32)            \
    X(5, 512, 16, 256, OP_C2R_4A, SK_COLS, 1, false, 1, 3, 1, 16, 32)                \
    /* hint variants of the multi-pass steps: split pass 0 (TWB 8) or more, \
       smaller CTAs per SM */                                                 \
    X(0, 1024, 8, 256, OP_R2C_4B, SK_ROWS_T, -1, false, 1, 2, 3, 32, 32)             \
    /* the split 2^19 = 1024 x 512: columns of 1024 (pass A), R2C pass B +  \
       post on rows of 512, C2C pass B on rows of 512 */                     \
    X(6, 1024, 8, 256, OP_C2C, SK_COLS, -1, true, 1, 3, 1, 32, 32)                   \
    X(7, 1024, 8, 256, OP_C2C, SK_COLS, 1, true, 1, 3, 1, 32, 32)                    \
    X(2, 512, 16, 256, OP_R2C_4B, SK_ROWS_T, -1, false, 1, 2, 1, 16, 32)             \
    X(3, 512, 16, 256, OP_R2C_4B, SK_ROWS_T, -1, false, 2, 1, 1, 16, 32)             \
    /* R2C pass B with the post-process on mirrored butterfly pairs (TWB 5): \
       rows of 512 (split 1024 x 512) and of 1024 (split 512 x 1024) */      \
    X(4, 512, 16, 256, OP_R2C_4B, SK_ROWS_T, -1, false, 1, 2, 5, 32, 16)             \
    X(5, 1024, 16, 512, OP_R2C_4B, SK_ROWS_T, -1, false, 1, 1, 5, 16, 4, 16)         \
    /* C2R pre-process + pass A on mirrored butterfly pairs (TWB 5) */       \
    X(6, 512, 16, 256, OP_C2R_4A, SK_COLS, 1, false, 1, 2, 5, 16, 32)                \
    X(7, 512, 16, 256, OP_C2R_4A, SK_COLS, 1, false, 1, 1, 5, 16, 32)                \
    X(4, 512, 16, 256, OP_C2C, SK_ROWS_T, 1, false, 1, 3, 1, 16, 32)                 \
    X(5, 512, 16, 256, OP_C2C, SK_ROWS_T, -1, false, 1, 3, 1, 16, 32)                \
    X(1, 1024, 4, 128, OP_R2C_4B, SK_ROWS_T, -1, false, 2, 3, 11, 32, 32)            \
    X(2, 512, 8, 128, OP_C2C, SK_COLS, -1, true, 2, 3, 9, 16, 32)                   \
    X(3, 512, 8, 128, OP_C2C, SK_COLS, 1, true, 2, 3, 9, 16, 32)                    \
    X(4, 1024, 4, 128, OP_C2C, SK_ROWS_T, -1, false, 2, 3, 9, 32, 32)                \
    X(5, 1024, 4, 128, OP_C2C, SK_ROWS_T, 1, false, 2, 3, 9, 32, 32)                 \
    X(6, 256, 16, 256, OP_C2C, SK_COLS, -1, true, 2, 3, 9, 16, 16)                   \
    X(7, 256, 16, 256, OP_C2C, SK_COLS, 1, true, 2, 3, 9, 16, 16)                    \
    /* C2C 4096 rows, 256 threads per transform: taken automatically by row  \
       steps of less than one wave of tiles (plan.cpp try_specialize) */     \
    X(6, 4096, 1, 256, OP_C2C, SK_ROWS, -1, false, 2, 2, 9, 16, 16, 16)              \
    X(7, 4096, 1, 256, OP_C2C, SK_ROWS, 1, false, 2, 2, 9, 16, 16, 16)               \
    X(0, 256, 16, 256, OP_C2C, SK_ROWS_T, -1, false, 2, 3, 9, 16, 16)                \
    X(1, 256, 16, 256, OP_C2C, SK_ROWS_T, 1, false, 2, 3, 9, 16, 16)                 \
    X(2, 256, 16, 256, OP_C2C, SK_COLS, -1, false, 2, 3, 9, 16, 16)                  \
    X(3, 256, 16, 256, OP_C2C, SK_COLS, 1, false, 2, 3, 9, 16, 16)                   \
    X(4, 2048, 4, 256, OP_C2C, SK_COLS, -1, false, 1, 3, 1, 16, 16, 8)               \
    X(5, 2048, 4, 256, OP_C2C, SK_COLS, 1, false, 1, 3, 1, 16, 16, 8)                \
    /* the C2R form with mirrored pairs in its split pass 0: a hint variant  \
       (slower than the plain split pass for N = 6000) */                   \
    X(6, 3000, 1, 128, OP_C2R_HALF, SK_ROWS, 1, false, 2, 4, 15, 15, 25, 8)          \
    X(7, 2187, 2, 192, OP_C2R_PAIR, SK_ROWS, 1, false, 2, 2, 15, 9, 9, 27)

#define SIP_SK_SHARDS 8
