// prime_field:: functions (reference src/linear_gkr/prime_field.cpp).
#include "linear_gkr/prime_field.h"
#include <cstdlib>
#include <stdlib.h>

namespace prime_field
{
const unsigned long long mod = 2305843009213693951ULL;
bool initialized = false;

void init() { initialized = true; }
void init_random() {}

static thread_local struct random_data *tl_state = nullptr;

void set_thread_random_state(struct random_data *state) { tl_state = state; }

int next_rand()
{
    if (tl_state) {
        int32_t r;
        random_r(tl_state, &r);
        return (int)r;
    }
    return rand();
}

// two draws, real part first (prime_field.cpp:35-41)
field_element random()
{
    field_element r;
    r.real = (unsigned long long)next_rand() % mod;
    r.img = (unsigned long long)next_rand() % mod;
    return r;
}

field_element random_real_only()
{
    field_element r;
    r.real = (unsigned long long)next_rand() % mod;
    r.img = 0;
    return r;
}

// the order-2^62 generator (real 2^31, img 1033321771269002680) squared
// 62 - log_order times (prime_field.cpp:60-73)
field_element get_root_of_unity(int log_order)
{
    assert(log_order <= 61);
    field_element r;
    r.real = 2147483648ULL;
    r.img = 1033321771269002680ULL;
    for (int i = 0; i < __max_order - log_order; ++i) r = r * r;
    return r;
}

field_element fast_pow(field_element x, __uint128_t p)
{
    field_element r(1);
    while (p) {
        if (p & 1) r = r * x;
        x = x * x;
        p >>= 1;
    }
    return r;
}

// x^(p^2 - 2)
field_element inv(field_element x)
{
    __uint128_t p = mod;
    return fast_pow(x, p * p - 2);
}
}  // namespace prime_field
