// Drop-in for the reference's fft_gkr side-prover binary (its main,
// src/VPD/fft_circuit_GKR.cpp:827-845): `fft_gkr <lg> <out>` proves the
// inverse-FFT circuit of size 2^lg on the GPU with the random stream of a
// fresh process (seed 1) and writes "v_time proof_size p_time" to <out>, the
// line the reference verifier reads back (vpd_verifier.cpp:89-99).  A run
// whose messages fail the in-process checks prints the reference's error line.
// VIRGO_DEVICE selects the GPU.
#include <cstdio>
#include <cstdlib>
#include "virgo_b200.h"

int main(int argc, char *argv[])
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <lg> <out>\n", argv[0]);
        return 2;
    }
    const int lg = atoi(argv[1]);
    const char *dev_env = getenv("VIRGO_DEVICE");
    vg_ctx *ctx = nullptr;
    vg_fft_gkr_stats st;
    if (vg_ctx_create(dev_env ? atoi(dev_env) : 0, &ctx) != VG_OK ||
        vg_fft_gkr_run(ctx, lg, 1, &st, nullptr, nullptr) != VG_OK) {
        fprintf(stderr, "fft_gkr: %s\n", vg_last_error());
        if (ctx) vg_ctx_destroy(ctx);
        return 1;
    }
    vg_ctx_destroy(ctx);
    if (!st.pass) fprintf(stderr, "Error, fft gkr failed\n");
    FILE *out = fopen(argv[2], "w");
    if (!out) return 1;
    fprintf(out, "%f %d %f\n", st.v_time, st.proof_size, st.p_time);
    fclose(out);
    return 0;
}
