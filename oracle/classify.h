/*
 * classify.h - boundary classification for the reference harness
 * (TEST INFRASTRUCTURE ONLY): LrsData::Init of anc-field/src/lrs-data.hpp:
 * 116-215 in C. Air cells 1..n-2 with solid face neighbours are sorted into
 * the 26 groups of lrs-data.hpp:53-78 (patterns :24-51), scan order z-y-x,
 * each point {x, y, z, material per solid neighbour in X_P, X_M, Y_P, Y_M,
 * Z_P, Z_M order}.
 */
#ifndef ORACLE_CLASSIFY_H
#define ORACLE_CLASSIFY_H
#include <stdint.h>

static int cls_faces(int g) { return g < 6 ? 1 : (g < 18 ? 2 : 3); }

/* decimal pattern of lrs-data.hpp:165-170 -> group, or -1 (lrs-data.hpp:327) */
static int cls_group(int pattern) {
    static const int pat[26] = {100000, 10000, 1000, 100, 10, 1,
                                101000, 100100, 100010, 100001, 11000, 10100, 10010, 10001,
                                1010, 1001, 110, 101,
                                101010, 101001, 100110, 100101, 11010, 11001, 10110, 10101};
    for (int g = 0; g < 26; ++g)
        if (pat[g] == pattern) return g;
    return -1;
}

static int cls_visit(const int32_t* v, int mx, int my, int mz, int64_t* cnt, int32_t** pos) {
    static const int weight[6] = {100000, 10000, 1000, 100, 10, 1};
    int64_t fill[26] = {0};
    for (int g = 0; g < 26; ++g)
        if (cnt) cnt[g] = 0;
    for (int z = 1; z < mz - 1; ++z)
        for (int y = 1; y < my - 1; ++y)
            for (int x = 1; x < mx - 1; ++x) {
                const int64_t i = ((int64_t)z * my + y) * mx + x;
                if (v[i] != -1) continue;
                const int32_t nb[6] = {v[i + 1], v[i - 1], v[i + mx], v[i - mx],
                                       v[i + (int64_t)mx * my], v[i - (int64_t)mx * my]};
                int pattern = 0, mats[3] = {-1, -1, -1}, k = 0;
                for (int d = 0; d < 6; ++d)
                    if (nb[d] != -1) {
                        pattern += weight[d];
                        if (k < 3) mats[k] = nb[d];
                        ++k;
                    }
                if (!pattern) continue;
                const int g = cls_group(pattern);
                if (g < 0) return -1;
                if (cnt) cnt[g]++;
                if (pos) {
                    const int w = 3 + cls_faces(g);
                    int32_t* o = pos[g] + fill[g] * w;
                    o[0] = x;
                    o[1] = y;
                    o[2] = z;
                    for (int f = 0; f < cls_faces(g); ++f) o[3 + f] = mats[f];
                    fill[g]++;
                }
            }
    return 0;
}

static int cls_count(const int32_t* v, int mx, int my, int mz, int64_t cnt[26]) {
    return cls_visit(v, mx, my, mz, cnt, 0);
}
static int cls_fill(const int32_t* v, int mx, int my, int mz, int32_t** pos) {
    return cls_visit(v, mx, my, mz, 0, pos);
}

#endif
