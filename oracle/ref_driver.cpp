// Oracle driver around the reference's own Stockham code, compiled on the
// CPU with ref_shim/ (test infrastructure only; built into oracle/_ref/ by
// oracle/Makefile when the reference sources are present).
//
// ref_stockham_c2c runs the reference's runStockhamForward
// (vendor/fft_stockham_mix.h:1218-1267) over coefficient tables built by
// the reference's BuildStockhamCoefficients (ops/include/params/
// fft_real_stockham.h:77-111).
#include <cstring>
#include <vector>

#include "fft_real_stockham.h"
#include "fft_stockham_mix.h"

extern "C" {

// Complex FFT of length m (2,3,5,7-smooth, m > 512 and not a power of two,
// the reference's Stockham admission) over `batch` interleaved rows.
// Returns 0, or -1 when the reference planner rejects the length.
int ref_stockham_c2c(long long m, int inverse, int batch, const float* in, float* out) {
    using namespace AsdSip;
    OpParam::FftRealStockham p{};
    p.fftN = (m % 2 == 1) ? m : 2 * m;
    p.batchSize = batch;
    p.isInverse = inverse ? 1 : 0;
    p.isC2R = 0;
    try {
        OpParam::RealStockhamPlan plan(p);
        if (plan.complexN != m) return -1;
        std::vector<float> dft = OpParam::BuildStockhamCoefficients(p, plan, 1);
        std::vector<float> tw = OpParam::BuildStockhamCoefficients(p, plan, 2);
        const size_t n = (size_t)batch * m * 2;
        std::vector<float> ws0(in, in + n), ws1(n);
        float* res = stockham::runStockhamForward(ws0.data(), ws1.data(), dft.data(), tw.data(), plan.radices.data(),
                                                  (int)plan.radices.size(), batch, (int)m);
        std::memcpy(out, res, n * sizeof(float));
    } catch (...) {
        return -1;
    }
    return 0;
}

}  // extern "C"
