// 8-bit child boxes relative to the parent box (node format SG_NODES_QUANT8).
//
// Per interior node and axis: origin = the smallest child lower bound, scale
// s = 2^e, the smallest power of two with 255 * s >= the node's extent. A child
// bound b is stored as a byte q with decode(q) = fl(origin + q * s) (q * s is
// exact, so one rounding, the same on host and device). Lower bounds round down
// and upper bounds round up until decode(q_lo) <= lo and decode(q_hi) >= hi
// hold in FP32, so every decoded box contains the FP32 box SORT tests.
//
// Why no hit is lost: the kernels run SORT's slab formula t = -o/d + b * (1/d)
// on the decoded bounds; it is monotonic in b under round-to-nearest, so the
// decoded box's slab interval contains SORT's interval for the exact box, and
// its entry distance is never larger. Every node SORT enters is entered, no
// node is culled that SORT keeps, and triangles are tested in FP32 unchanged.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "builder.h"
#include "layout.h"

namespace sg {
namespace {

inline float decode(uint32_t q, float s, float origin) { return origin + float(q) * s; }

// Smallest e in [-126, 127] with 255 * 2^e >= extent.
int exponent_for(double extent) {
    if (!(extent > 0.0)) return -126;
    int e = int(std::ceil(std::log2(extent / 255.0)));
    if (e < -126) e = -126;
    while (e < 127 && 255.0 * std::ldexp(1.0, e) < extent) ++e;
    return e;
}

bool quantize_axis(const float* lo, const float* hi, const int32_t* child, int W, float origin, int e, uint8_t* qlo,
                   uint8_t* qhi) {
    const float s = std::ldexp(1.0f, e);
    for (int j = 0; j < W; ++j) {
        if (child[j] == kEmptyRef) {  // inverted box: missed by every ray with finite origin and direction
            qlo[j] = 255;
            qhi[j] = 0;
            continue;
        }
        double fl = std::floor((double(lo[j]) - double(origin)) / double(s));
        double fh = std::ceil((double(hi[j]) - double(origin)) / double(s));
        int64_t a = int64_t(fl < 0.0 ? 0.0 : fl), b = int64_t(fh < 0.0 ? 0.0 : fh);
        if (a > 255) a = 255;
        while (a > 0 && decode(uint32_t(a), s, origin) > lo[j]) --a;
        if (decode(uint32_t(a), s, origin) > lo[j]) return false;
        if (b > 255) return false;
        while (b < 255 && decode(uint32_t(b), s, origin) < hi[j]) ++b;
        if (decode(uint32_t(b), s, origin) < hi[j]) return false;
        qlo[j] = uint8_t(a);
        qhi[j] = uint8_t(b);
    }
    return true;
}

}  // namespace

void quantize_nodes(const BuiltTree& t, std::vector<float4>& out) {
    const int W = t.width;
    const int f4 = W == 8 ? kQ8F4W8 : kQ8F4W4;
    const int64_t nn = t.interior();
    out.assign(size_t(nn > 0 ? nn : 1) * f4, float4{0.0f, 0.0f, 0.0f, 0.0f});
    for (int64_t k = 0; k < nn; ++k) {
        const int32_t* child = &t.child[size_t(k) * W];
        unsigned char* base = reinterpret_cast<unsigned char*>(&out[size_t(k) * f4]);
        float origin[3];
        uint32_t ebits = 0;
        uint8_t q[3][2][8];
        std::memset(q, 0, sizeof(q));
        for (int a = 0; a < 3; ++a) {
            const float* lo = &t.lo[(size_t(k) * 3 + a) * W];
            const float* hi = &t.hi[(size_t(k) * 3 + a) * W];
            float mn = FLT_MAX, mx = -FLT_MAX;
            for (int j = 0; j < W; ++j)
                if (child[j] != kEmptyRef) {
                    mn = lo[j] < mn ? lo[j] : mn;
                    mx = hi[j] > mx ? hi[j] : mx;
                }
            if (mn > mx) mn = mx = 0.0f;  // no children (never built, kept safe)
            origin[a] = mn;
            int e = exponent_for(double(mx) - double(mn));
            while (!quantize_axis(lo, hi, child, W, mn, e, q[a][0], q[a][1])) {
                if (++e > 127) throw std::runtime_error("child box cannot be quantised");
            }
            ebits |= uint32_t(e + 127) << (8 * a);
        }
        float* hdr = reinterpret_cast<float*>(base);
        hdr[0] = origin[0];
        hdr[1] = origin[1];
        hdr[2] = origin[2];
        std::memcpy(&hdr[3], &ebits, 4);
        if (W == 8) {
            for (int a = 0; a < 3; ++a) {
                std::memcpy(base + 16 * (1 + a), q[a][0], 8);
                std::memcpy(base + 16 * (1 + a) + 8, q[a][1], 8);
            }
            std::memcpy(base + 64, child, 32);
        } else {
            std::memcpy(base + 16, q[0][0], 4);
            std::memcpy(base + 20, q[0][1], 4);
            std::memcpy(base + 24, q[1][0], 4);
            std::memcpy(base + 28, q[1][1], 4);
            std::memcpy(base + 32, q[2][0], 4);
            std::memcpy(base + 36, q[2][1], 4);
            std::memcpy(base + 48, child, 16);
        }
    }
}

}  // namespace sg
