// Small integer helpers with the reference's names (include/infrastructure/utility.h:1-3).
#pragma once
int mylog(long long x);   // log2 of a power of two; aborts otherwise
int min(int x, int y);
int max(int x, int y);
