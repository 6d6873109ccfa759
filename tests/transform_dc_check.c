/* CPU check of the residual transforms exported by libtcodec_b200.so and
 * of the DC-only helpers in include/tcodec_b200_common.h, after the
 * reference's transform test (test/test_tcodec.c:3074-3149): DC gains of
 * the WHT and DCTs, the round-trip error bound on residual blocks within
 * +-2000, and the DC-only inverse helpers equal to the full inverse
 * transforms for every DC value in [-2000, 2000], negative rounding
 * included.  Built and run by tests/test_common_abi.py; exit status 0 when
 * every check holds. */
#include <stdio.h>
#include <string.h>

#include "tcodec_b200_common.h"

int main(void) {
    tc_coeff_t in[64], fwd[64], rec[64];
    int fail = 0;
    for (int i = 0; i < 16; i++) in[i] = 100;
    tc_fwht4x4(in, 4, fwd);
    fail += fwd[0] != 400;
    tc_iwht4x4(fwd, rec, 4);
    for (int i = 0; i < 16; i++) fail += rec[i] != 100;
    tc_fdct4x4_res(in, 4, fwd);
    fail += fwd[0] != 400;
    tc_idct4x4_res(fwd, rec, 4);
    for (int i = 0; i < 16; i++) fail += rec[i] < 99 || rec[i] > 101;
    for (int i = 0; i < 64; i++) in[i] = 100;
    tc_fdct8x8_res(in, 8, fwd);
    fail += fwd[0] != 800;
    tc_idct8x8_res(fwd, rec, 8);
    for (int i = 0; i < 64; i++) fail += rec[i] < 99 || rec[i] > 101;
    printf("dc gains / roundtrips: %d failures\n", fail);

    unsigned long long s = 12345;
    int bound = 0;
    for (int rep = 0; rep < 256; rep++) {
        for (int i = 0; i < 64; i++) {
            s = s * 6364136223846793005ULL + 1442695040888963407ULL;
            in[i] = (tc_coeff_t)((int)((s >> 33) % 4001) - 2000);
        }
        tc_fdct4x4_res(in, 4, fwd);
        tc_idct4x4_res(fwd, rec, 4);
        for (int i = 0; i < 16; i++) bound += in[i] - rec[i] > 2 || rec[i] - in[i] > 2;
        tc_fdct8x8_res(in, 8, fwd);
        tc_idct8x8_res(fwd, rec, 8);
        for (int i = 0; i < 64; i++) bound += in[i] - rec[i] > 2 || rec[i] - in[i] > 2;
    }
    printf("round-trip bound: %d samples off by more than 2\n", bound);

    int dcfail = 0;
    for (int dc = -2000; dc <= 2000; dc++) {
        memset(in, 0, sizeof(in));
        in[0] = (tc_coeff_t)dc;
        tc_idct4x4_res(in, rec, 4);
        for (int i = 0; i < 16; i++) dcfail += rec[i] != tc_idct_dc4_res(dc);
        memset(in, 0, sizeof(in));
        in[0] = (tc_coeff_t)dc;
        tc_idct8x8_res(in, rec, 8);
        for (int i = 0; i < 64; i++) dcfail += rec[i] != tc_idct_dc8_res(dc);
    }
    printf("dc-only helpers: %d mismatching samples\n", dcfail);
    return (fail || bound || dcfail) ? 1 : 0;
}
