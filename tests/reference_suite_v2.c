/*
 * reference_suite_v2.c: the reference's own C regression tests, run
 * against whichever library this file is linked with.
 *
 * The test functions of the reference suite (test/test_tcodec.c of the
 * reference tree) are `static`, so this file includes the suite itself with
 * its main() renamed and calls the tests that exercise the v2 bitstream and
 * the modules beneath it, then prints the suite's own pass tally.  Its
 * exit status is 0 only when every one of them passed.
 *
 * Left out: the tests whose encoders are created from tc_config_defaults()
 * alone or that switch to the v0 / v1 bitstream (test/test_tcodec.c:105-1051
 * outside the v2 tests, 1230-1282, 1282-1560, 1726-2470, 2470-3074): those
 * configurations select the legacy block bitstream, which this library
 * rejects at encoder creation by design.
 *
 * Built by oracle/Makefile (target `suite`) twice: linked with
 * libtcodec_b200.so (oracle/_ref/test_v2_suite_b200) and with the reference
 * library's own objects (oracle/_ref/test_v2_suite_ref), so the same tests
 * are shown to pass on both.
 */
#define main reference_suite_main
#include "test/test_tcodec.c"
#undef main

int main(void)
{
    printf("reference C suite, v2 and module tests\n");

    /* module tests (test/test_tcodec.c:84-193) */
    test_version();
    test_error_strings();
    test_color_roundtrip();
    test_config_defaults();
    test_decoder_create_destroy();

    /* v2 encoder / decoder tests */
    test_v2_multiref();        /* :811  */
    test_v2_cfl();             /* :869  */
    test_v2_bframes();         /* :946  */
    test_v2_roundtrip();       /* :1063 */
    test_v2_fast_presets();    /* :1147 */
    test_fuzz_malformed_v2();  /* :1560 */
    test_v2_sao();             /* :3545 */

    /* range coder and transforms (:3074-3545) */
    test_rc_engine_roundtrip();
    test_rc_context_model();
    test_rc_coeff_coding();
    test_transform_roundtrip();

    printf("  Results: %d/%d passed", g_tests_passed, g_tests_run);
    if (g_tests_failed > 0)
        printf(", %d FAILED", g_tests_failed);
    printf("\n");
    return g_tests_failed > 0 ? 1 : 0;
}
