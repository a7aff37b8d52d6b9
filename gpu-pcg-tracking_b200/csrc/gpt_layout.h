// gpt_layout.h -- the part layout of the partitioned PCG (pcg_quad_kernel): which knots each of
// the four factoring warps owns and where the separator knots lie.  Plain C++ (host and device), so
// the CPU tests compile it and check the layout for every horizon.
#pragma once

#if defined(__CUDACC__)
#define GPT_HD __host__ __device__
#else
#define GPT_HD
#endif

namespace gpt {

constexpr int QUAD_NWARP = 4;

struct QuadLayout {
    int P;
    int a[QUAD_NWARP], b[QUAD_NWARP];  // part p: knots a[p] .. b[p] (b[p] < a[p]: empty)
    int s[QUAD_NWARP - 1];             // separator knots
};
GPT_HD inline QuadLayout quad_layout(int n)
{
    QuadLayout L;
    int P = QUAD_NWARP;
    if (n < 2 * P) {
        P = (n + 1) / 2;
        P = P < 1 ? 1 : (P > QUAD_NWARP ? QUAD_NWARP : P);
    }
    L.P = P;
    const int nint = n - (P - 1);
    int len[QUAD_NWARP] = {0, 0, 0, 0};
    if (P == 1) {
        len[0] = n;
    } else if (P == 2) {
        len[0] = nint / 2;
        len[1] = nint - len[0];
    } else {
        const int y = (10 * nint) / (26 + 10 * (P - 2));  // edge parts weighted 1.3
        const int rest = nint - (P - 2) * y;
        len[0] = rest / 2;
        for (int p = 1; p < P - 1; ++p) len[p] = y;
        len[P - 1] = rest - len[0];
    }
    int pos = 0;
    for (int p = 0; p < QUAD_NWARP; ++p) {
        L.a[p] = pos;
        L.b[p] = pos + (p < P ? len[p] : 0) - 1;
        pos += p < P ? len[p] : 0;
        if (p < QUAD_NWARP - 1) {
            L.s[p] = pos;
            if (p < P - 1) ++pos;
        }
    }
    return L;
}

}  // namespace gpt
