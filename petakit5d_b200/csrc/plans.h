// Compile-time transform plans.  Each entry is a transform length and its radix sequence; the pass
// kernels are instantiated once per entry, so every stage runs with constant radix, stride and
// twiddle step (straight-line code, no register spills).  Lengths without an entry use plan 0,
// the runtime-radix engine (any length, slower).
#pragma once

#define PK_THREADS 256        // threads per pass CTA
#define PK_TILE_POINTS 4096   // complex points one CTA holds (16 per thread)

struct PlanDef {
    int n;
    int nst;
    int rad[8];
};

// Radices 2/3/4/5/8/16 have register butterflies; 7, 9, 11, 13, 17 run as unrolled direct DFTs.
constexpr PlanDef kPlans[] = {
    {0, 0, {0}},                  // 0: runtime engine
    {1, 0, {0}},
    {2, 1, {2}},
    {4, 1, {4}},
    {8, 1, {8}},
    {16, 1, {16}},
    {32, 2, {16, 2}},
    {64, 2, {16, 4}},
    {128, 2, {16, 8}},
    {256, 2, {16, 16}},
    {512, 3, {16, 16, 2}},
    {1024, 3, {16, 16, 4}},
    {2048, 3, {16, 16, 8}},
    {4096, 3, {16, 16, 16}},
    {48, 2, {16, 3}},
    {80, 2, {16, 5}},
    {96, 3, {16, 2, 3}},
    {112, 2, {16, 7}},
    {144, 2, {16, 9}},
    {160, 3, {16, 2, 5}},
    {176, 2, {16, 11}},
    {180, 3, {4, 9, 5}},
    {192, 3, {16, 4, 3}},
    {208, 2, {16, 13}},
    {210, 4, {2, 3, 5, 7}},
    {224, 3, {16, 2, 7}},
    {240, 3, {16, 3, 5}},
    {272, 2, {16, 17}},
    {288, 3, {16, 2, 9}},
    {320, 3, {16, 4, 5}},
    {352, 3, {16, 2, 11}},
    {360, 3, {8, 9, 5}},
    {384, 3, {16, 8, 3}},
    {416, 3, {16, 2, 13}},
    {420, 4, {4, 3, 5, 7}},
    {448, 3, {16, 4, 7}},
    {480, 4, {16, 2, 3, 5}},
    {544, 3, {16, 2, 17}},
    {576, 3, {16, 4, 9}},
    {640, 3, {16, 8, 5}},
    {720, 3, {16, 9, 5}},
    {768, 3, {16, 16, 3}},
    {960, 4, {16, 4, 3, 5}},
    {1152, 3, {16, 8, 9}},
    {1280, 3, {16, 16, 5}},
    {1536, 4, {16, 16, 2, 3}},
};
constexpr int kNumPlans = sizeof(kPlans) / sizeof(kPlans[0]);

constexpr int plan_product(int p) {
    int v = 1;
    for (int i = 0; i < kPlans[p].nst; i++) v *= kPlans[p].rad[i];
    return v;
}

constexpr int plan_ns_before(int p, int s) {
    int v = 1;
    for (int i = 0; i < s; i++) v *= kPlans[p].rad[i];
    return v;
}
constexpr bool direct_radix(int r) { return !(r == 2 || r == 3 || r == 4 || r == 5 || r == 8 || r == 16); }

// Stage-ordered twiddle table of a compile-time plan: stage s (radix R, stride NS > 1) holds
// W_N^{r k N/(NS R)} at [off_s + (r-1) NS + k] (r = 1..R-1, k < NS), so the threads of a warp read
// consecutive entries; a direct-DFT radix appends its R roots W_R^e.  The table has N - 1 + (the
// direct radices) entries.
constexpr int stage_tw_size(int p, int s) {
    const int ns = plan_ns_before(p, s), r = kPlans[p].rad[s];
    return (ns > 1 ? (r - 1) * ns : 0) + (direct_radix(r) ? r : 0);
}
constexpr int stage_tw_off(int p, int s) {
    int o = 0;
    for (int i = 0; i < s; i++) o += stage_tw_size(p, i);
    return o;
}
constexpr int plan_tw_size(int p) { return stage_tw_off(p, kPlans[p].nst); }

// Shared-memory slots reserved for an axis table of length-n transforms (root table of n entries
// for the runtime engine, stage-ordered table otherwise).
#define PK_TW_EXTRA 32
__host__ __device__ constexpr int tw_slots(int n) { return n + PK_TW_EXTRA; }

// Lines (y pass, contiguous) and columns (x/z passes, a power of two for sector-aligned rows) per tile.
constexpr int plan_lines_y(int n, int tp = PK_TILE_POINTS) { return n >= 1 ? (tp / n > 0 ? tp / n : 1) : 1; }
constexpr int plan_cols_xz(int n, int tp = PK_TILE_POINTS) {
    int t = 1;
    while (t * 2 * n <= tp) t *= 2;
    return t;
}

// Small tiles (1024 points, same 256 threads) for volumes too small to fill the GPU with 4096-point
// tiles: four times the CTAs, at the cost of idle threads in the wide stages.  Instantiated for the
// compile-time plans up to length 256.
#define PK_TILE_SMALL 1024
constexpr bool small_tile_plan(int p) { return p > 0 && kPlans[p].nst >= 2 && kPlans[p].n <= 256; }

inline int pk_find_plan(int n) {
    for (int p = 1; p < kNumPlans; p++)
        if (kPlans[p].n == n && plan_product(p) == n) return p;
    return 0;
}
