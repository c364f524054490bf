// In-memory layered circuit with the reference's layout
// (include/linear_gkr/circuit_fast_track.h:6-57).  The reference verifier's
// read_circuit fills these objects directly, so names, member types and
// order are kept as they are; the prover copies them to the device in
// zk_prover::get_circuit.
#ifndef __circuit
#define __circuit
#include <unordered_map>
#include <utility>
#include <vector>
#include "linear_gkr/prime_field.h"

class gate
{
public:
    int ty;
    long long u, v;
    gate() {}
    gate(int t, long long U, long long V)
    {
        ty = t, u = U, v = V;
    }
};

class layer
{
public:
    gate *gates;
    int bit_length;
    std::unordered_map<int, std::vector<std::pair<int, std::pair<int, int> > > > u_gates;
    std::unordered_map<int, std::vector<std::pair<int, std::pair<int, int> > > > v_gates;
    bool is_parallel;
    int block_size;
    int log_block_size;
    int repeat_num;
    int log_repeat_num;
    layer()
    {
        is_parallel = false;
        gates = NULL;
        bit_length = 0;
    }
    ~layer() {}
};

class layered_circuit
{
public:
    layer *circuit;
    int total_depth;
    layered_circuit()
    {
        circuit = NULL;
        total_depth = 0;
    }
    ~layered_circuit() {}
};

#endif
