// reference src/infrastructure/utility.cpp
#include "infrastructure/utility.h"
#include <cstdio>
#include <cstdlib>

int mylog(long long x)
{
    for (int i = 0; i < 64; ++i)
        if ((1LL << i) == x) return i;
    fprintf(stderr, "mylog: %lld is not a power of two\n", x);
    abort();
}
int min(int x, int y) { return x > y ? y : x; }
int max(int x, int y) { return x > y ? x : y; }
