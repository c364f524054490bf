// F_{p^2}, p = 2^61 - 1, with the reference's interface
// (include/linear_gkr/prime_field.h, src/linear_gkr/prime_field.cpp): namespace
// prime_field, class field_element {img, real} with + - * and unary -, the
// 2-adic roots of unity, inverse, fast_pow and random().  Arithmetic is exact
// and every result canonical, as in the reference, so values agree bit for bit.
// Written portably (128-bit products) instead of with x86 inline assembly.
#pragma once
#ifndef __prime_field
#define __prime_field

#include "infrastructure/constants.h"
#include <cassert>
#include <cstring>
#include <memory>
#include <vector>

struct random_data;

namespace prime_field
{
extern bool initialized;
extern const unsigned long long mod;

void init();
void init_random();

// x mod p for x < 2^64 up to one extra p (the reference's myMod)
inline unsigned long long myMod(unsigned long long x) { return (x >> 61) + (x & 2305843009213693951ULL); }
// x * y folded once mod p, result below 2p for x, y < 2^62 (the reference's mymult)
inline unsigned long long mymult(const unsigned long long x, const unsigned long long y)
{
    unsigned __int128 t = (unsigned __int128)x * y;
    unsigned long long lo = (unsigned long long)t, hi = (unsigned long long)(t >> 64);
    return ((hi << 3) | (lo >> 61)) + (lo & 2305843009213693951ULL);
}

class field_element
{
public:
    unsigned long long img, real;

    std::unique_ptr<char[]> bit_stream()
    {
        char *p = new char[sizeof(field_element)];
        memcpy(p, this, sizeof(field_element));
        return std::unique_ptr<char[]>(p);
    }
    int size() { return sizeof(field_element); }

    inline field_element() : img(0), real(0) {}
    inline field_element(const unsigned long long x) : img(0), real(x % 2305843009213693951ULL) {}

    static inline unsigned long long red(unsigned __int128 x)
    {
        const unsigned long long P = 2305843009213693951ULL;
        unsigned long long r = (unsigned long long)(x & P) + (unsigned long long)(x >> 61);
        r = (r & P) + (r >> 61);
        return r >= P ? r - P : r;
    }
    inline field_element operator+(const field_element &b) const
    {
        const unsigned long long P = 2305843009213693951ULL;
        field_element r;
        r.real = real + b.real;
        r.img = img + b.img;
        if (r.real >= P) r.real -= P;
        if (r.img >= P) r.img -= P;
        return r;
    }
    inline field_element operator-(const field_element &b) const
    {
        const unsigned long long P = 2305843009213693951ULL;
        field_element r;
        r.real = real >= b.real ? real - b.real : real + P - b.real;
        r.img = img >= b.img ? img - b.img : img + P - b.img;
        return r;
    }
    inline field_element operator-() const
    {
        const unsigned long long P = 2305843009213693951ULL;
        field_element r;
        r.real = real ? P - real : 0;
        r.img = img ? P - img : 0;
        return r;
    }
    // (a + bi)(c + di) = (ac - bd) + (ad + bc)i, each part reduced once from 123 bits
    inline field_element operator*(const field_element &b) const
    {
        const unsigned long long P = 2305843009213693951ULL;
        field_element r;
        unsigned __int128 re = (unsigned __int128)real * b.real + (unsigned __int128)(img ? P - img : 0) * b.img;
        unsigned __int128 im = (unsigned __int128)real * b.img + (unsigned __int128)img * b.real;
        r.real = red(re);
        r.img = red(im);
        return r;
    }
    bool operator==(const field_element &b) const { return real == b.real && img == b.img; }
    bool operator!=(const field_element &b) const { return !(*this == b); }
};

const int __max_order = 62;
field_element get_root_of_unity(int order);   // root of order 2^order
field_element random_real_only();
field_element random();
field_element fast_pow(field_element x, __uint128_t p);
field_element inv(field_element x);

// Randomness source.  random() draws two values from glibc rand(), as the
// reference does (prime_field.cpp:35-41).  A thread can instead draw from its
// own glibc random_r state (identical sequence to srand(seed)/rand() when it was
// initialised with initstate_r(seed, buf, 128, .)), which lets independent
// proofs run concurrently with reproducible transcripts.
void set_thread_random_state(struct random_data *state);
int next_rand();
}  // namespace prime_field
#endif
