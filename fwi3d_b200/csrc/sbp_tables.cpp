// Expands the SBP coefficient tables used by sbp.cuh.
//
// The weights are the rationals of the 4th-order SBP operators the reference
// discretises with (nmbader/fwi3d spatial_operators.cpp:181 for D1,
// spatial_operators.hpp:37-43 for D2var, :241 for S, spatial_operators.cpp:15
// for H); each is rounded to float from its double-precision rational exactly
// as the reference's `data_t` initialisers are, so both codes use identical
// single-precision coefficients.
#include <cstring>
#include <mutex>
#include "sbp.cuh"

namespace fwi {

SbpTables g_sbp_host;

namespace {
inline float q(double p, double r) { return (float)(p / r); }
}  // namespace

namespace {
void build_sbp_tables()
{
    SbpTables t;
    std::memset(&t, 0, sizeof(t));

    // Interior D2var: weight groups for u(i), u(i-1)/u(i+1), u(i-2)/u(i+2).
    const double d2in[10][2] = {{-3, 4}, {-5, 6}, {-1, 24}, {1, 6}, {1, 2},
                                {1, 2},  {1, 6},  {-1, 8},  {1, 6}, {-1, 8}};
    for (int i = 0; i < 10; i++) t.d2in[i] = q(d2in[i][0], d2in[i][1]);

#define D2B(r, j, k, p, d) t.d2b[r][j][k] = q((double)(p), (double)(d));
#include "sbp_d2_closure.inc"
#undef D2B

    // D1 closure rows (4 x 6), written as (numerator, denominator).
    const double d1b[4][6][2] = {
        {{-24, 17}, {59, 34}, {-4, 17}, {-3, 34}, {0, 1}, {0, 1}},
        {{-1, 2}, {0, 1}, {1, 2}, {0, 1}, {0, 1}, {0, 1}},
        {{4, 43}, {-59, 86}, {0, 1}, {59, 86}, {-4, 43}, {0, 1}},
        {{3, 98}, {0, 1}, {-59, 98}, {0, 1}, {32, 49}, {-4, 49}},
    };
    for (int r = 0; r < 4; r++)
        for (int j = 0; j < 6; j++) t.d1b[r][j] = q(d1b[r][j][0], d1b[r][j][1]);
    t.d1c0 = q(2, 3);
    t.d1c1 = q(-1, 12);

    t.sb[0] = q(11, 6);
    t.sb[1] = -3.f;
    t.sb[2] = 1.5f;
    t.sb[3] = q(-1, 3);

    t.hq[0] = q(17, 48);
    t.hq[1] = q(59, 48);
    t.hq[2] = q(43, 48);
    t.hq[3] = q(49, 48);

    g_sbp_host = t;
}
}  // namespace

// Built once per process: engines are created on several host threads (the
// serving loop's workers), so the table is written under std::call_once,
// whose completion every later caller observes before reading it.
void init_sbp_tables()
{
    static std::once_flag once;
    std::call_once(once, build_sbp_tables);
}

}  // namespace fwi
