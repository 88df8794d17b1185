"""Case lists of the reference's device unit tests (hicann/sip), as
(batch, n, direction) / 2D / 3D tuples.  Inputs of those tests come from
the fixed-seed LCG (oracle.ut_input) and are compared with numpy.fft
goldens under isclose(rtol=1e-3, atol=1e-5).

Sources (relative to the reference root):
  C2C 1D  tests/ut/unittest/fft/1d/c2c/test_fft_c2c_1d.cpp:165-226
  R2C 1D  tests/ut/unittest/fft/1d/r2c/test_fft_r2c_1d.cpp:161-207
  C2R 1D  tests/ut/unittest/fft/1d/c2r/test_fft_c2r_1d.cpp:161-185
  C2C 2D  tests/ut/unittest/fft/2d/c2c/test_fft_c2c_2d.cpp:144-166
  C2C 3D  tests/ut/unittest/fft/3d/c2c/test_fft_c2c_3d.cpp:143-150
"""
F, I = 0x10, 0x11

C2C_1D = [(1, n, F) for n in (64, 81, 125, 49, 121, 169, 17, 19, 1024, 729, 625, 343, 289, 361, 4096, 6561, 32768,
                              4620, 210, 2310, 143, 323, 360)] + [(2, 1024, F), (2, 210, F)] + \
         [(1, n, I) for n in (64, 81, 125, 49, 121, 169, 17, 19, 1024, 729, 625, 343, 289, 361, 4096, 32768, 4620,
                              210, 2310)] + [(2, 1024, I)]

R2C_1D = [(1, 16, F), (1, 27, F), (1, 25, F), (1, 49, F), (1, 121, F), (1, 169, F), (1, 289, F), (1, 361, F),
          (1, 210, F), (2, 16, F), (4, 27, F), (8, 210, F), (1, 2048, F), (1, 2187, F), (1, 3125, F), (1, 2401, F),
          (2, 1573, F), (1, 2160, F), (1, 32768, F), (1, 2520, F)] + \
         [(1, n, I) for n in (16, 27, 25, 49, 121, 169, 289, 361, 210)] + [(2, 16, I)] + \
         [(1, n, I) for n in (2048, 2187, 3125, 2401)] + [(2, 1573, I), (1, 2160, I), (1, 32768, I)]

C2R_1D = [(1, 16, F), (2, 32, F), (1, 64, F), (1, 27, F), (1, 25, F), (1, 49, F), (1, 121, F), (1, 169, F),
          (1, 289, F), (1, 361, F), (1, 30, F), (1, 210, F), (2, 30, F), (1, 2048, F), (1, 2187, F), (1, 3125, F),
          (1, 2401, F), (2, 1573, F), (1, 2160, F), (1, 32768, F), (1, 2520, F)] + \
         [(1, n, I) for n in (16, 27, 25, 49, 121, 169, 289, 361, 30, 210)] + [(2, 16, I)] + \
         [(1, n, I) for n in (2048, 2187, 3125, 2401)] + [(2, 1573, I), (2, 1056, I), (1, 2160, I), (1, 32768, I)]

# (x, y, batch, direction)
C2C_2D = [(64, 64, 1, F), (64, 64, 1, I), (128, 256, 1, F), (32, 48, 2, F), (112, 104, 1, F), (500, 50, 2, F),
          (500, 50, 2, I)]

# (x, y, z, batch, direction)
C2C_3D = [(8, 8, 8, 1, F), (16, 16, 16, 2, I), (48, 40, 24, 1, F)]
