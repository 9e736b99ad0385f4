// rzk_hostutil.h - host-side pieces shared by the clustering and LightSlice builders:
// the reference's discrete distribution and its Random::operator() on the counter-based
// stream.
#ifndef RZK_HOSTUTIL_H_
#define RZK_HOSTUTIL_H_

#include <cstdint>
#include <vector>

#include "rzk_math.cuh"

namespace rzk {

struct DPdf {   // DiscretePdf (pdf.cc:18-77)
    std::vector<float> pdf, cdf;
    bool monotone = true;
    void set(const float *a, int n) {
        pdf.assign(n, 0.0f);
        cdf.assign(n, 0.0f);
        if (n == 0) return;
        float sum = 0.0f;
        for (int i = 0; i < n; ++i) sum += a[i];
        if (sum == 0.0f) return;
        for (int i = 0; i < n; ++i) pdf[i] = a[i] / sum;
        cdf[0] = pdf[0];
        for (int i = 1; i < n; ++i) cdf[i] = cdf[i - 1] + pdf[i];
        cdf[n - 1] = 1.0f;
        for (int i = 1; i < n; ++i)
            if (cdf[i] < cdf[i - 1]) { monotone = false; break; }
    }
    // first i with v < cdf[i] (linear scan semantics; a binary search where the cdf is
    // non-decreasing finds the same index)
    void sample(float v, int &k, float &pk) const {
        int n = (int)cdf.size();
        if (monotone) {
            int lo = 0, hi = n;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (v < cdf[mid]) hi = mid; else lo = mid + 1;
            }
            if (lo < n) { k = lo; pk = pdf[lo]; return; }
        } else {
            for (int i = 0; i < n; ++i)
                if (v < cdf[i]) { k = i; pk = pdf[i]; return; }
        }
        k = -1;
        pk = 0.0f;
    }
};

struct HostRng {   // Random::operator() on the counter-based stream (random.h:60-63)
    uint32_t seed, stream, path, d = 0;
    float next() {
        uint4 blk = philox4x32_10(make_uint4(d >> 2, path, stream, 0x52454e5au), seed, 0x4b5a4f52u);
        uint32_t w = (d & 3) == 0 ? blk.x : ((d & 3) == 1 ? blk.y : ((d & 3) == 2 ? blk.z : blk.w));
        d++;
        return (w & 0x00ffffffu) * (1.0f / 16777216.0f);
    }
};


}  // namespace rzk

#endif  // RZK_HOSTUTIL_H_
