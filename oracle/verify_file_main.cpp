// A verifier process for a serialized GPU proof.  TEST INFRASTRUCTURE ONLY.
//
//   zk_verify_file <circuit.txt> <meta.txt> <proof file> <result.txt>
//
// The reference verifier (src/linear_gkr/zk_verifier.cpp and
// src/VPD/vpd_verifier.cpp, compiled unchanged) drives the drop-in prover
// classes, whose device calls are answered from the proof file written by
// vg_session_write_proof (oracle/replay_abi.cpp): no GPU and no prover work
// in this process.  It seeds rand() with the proof's seed, as the proving
// session did, so the verifier draws the challenges the proof was made for.
// Prints Pass only when the verifier accepts and the proof file was used up.
#include "linear_gkr/zk_verifier.h"
#include "linear_gkr/zk_prover.h"
#include "linear_gkr/prime_field.h"
#include <cstdio>
#include <cstdlib>

extern "C" int vg_replay_open(const char *path, unsigned *seed);
extern "C" int vg_replay_close(void);
extern "C" const char *vg_last_error(void);

static zk_verifier g_verifier;
static zk_prover g_prover;

int main(int argc, char **argv)
{
    if (argc != 5) {
        fprintf(stderr, "usage: %s circuit meta proof result\n", argv[0]);
        return 2;
    }
    unsigned seed = 0;
    if (vg_replay_open(argv[3], &seed) != 0) {
        fprintf(stderr, "zk_verify_file: %s\n", vg_last_error());
        return 2;
    }
    srand(seed);
    prime_field::init();
    g_prover.total_time = 0;
    g_prover.quiet = true;
    g_verifier.get_prover(&g_prover);
    g_verifier.read_circuit(argv[1], argv[2]);
    g_prover.get_circuit(g_verifier.C);
    const bool ok = g_verifier.verify(argv[4]);
    const int rc = vg_replay_close();
    if (rc != 0) fprintf(stderr, "zk_verify_file: %s\n", vg_last_error());
    printf("%s\n", ok && rc == 0 ? "Pass" : "Fail");
    fflush(stdout);
    return ok && rc == 0 ? 0 : 1;
}
