// Driver for the oracle prover binaries.  TEST INFRASTRUCTURE ONLY.
//
//   <binary> <circuit.txt> <meta.txt> <result.txt> <seed> [transcript.bin]
//
// It plays the role of the reference CLI (src/linear_gkr/main_zk.cpp:11-26)
// with one addition: srand(seed) before anything draws randomness, so that a
// proof is reproducible.  The reference seeds nothing, which is glibc's seed 1.
// Compiled against the reference headers it gives the CPU reference prover;
// compiled against this repository's drop-in headers and linked to the GPU
// prover it gives the acceptance run (the verifier sources are unchanged).
#include "linear_gkr/zk_verifier.h"
#include "linear_gkr/zk_prover.h"
#include "linear_gkr/prime_field.h"
#include <cstdio>
#include <cstdlib>

extern "C" void virgo_transcript_open(const char *path);
extern "C" void virgo_transcript_close();

static zk_verifier g_verifier;
static zk_prover g_prover;

int main(int argc, char **argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s circuit meta result seed [transcript]\n", argv[0]);
        return 2;
    }
    srand((unsigned)strtoul(argv[4], nullptr, 10));
    virgo_transcript_open(argc > 5 ? argv[5] : nullptr);
    prime_field::init();
    g_prover.total_time = 0;
    g_verifier.get_prover(&g_prover);
    g_verifier.read_circuit(argv[1], argv[2]);
    g_prover.get_circuit(g_verifier.C);
    bool ok = g_verifier.verify(argv[3]);
    virgo_transcript_close();
    printf("%s\n", ok ? "Pass" : "Fail");
    fflush(stdout);
    return ok ? 0 : 1;
}
