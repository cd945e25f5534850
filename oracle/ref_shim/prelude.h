// Forced-include prelude for compiling reference sources with g++ on Linux.
// Supplies the MSVC-isms those sources lean on (implicit <cstring>, min/max
// overloads over mixed unsigned/int arguments).  Test infrastructure only.
#ifndef RB2_ORACLE_PRELUDE_H
#define RB2_ORACLE_PRELUDE_H
#include <cstring>
#include <cstdint>
#include <cstdio>
#include <cfloat>
#include <algorithm>
#include <exception>
using std::exception;
inline unsigned int max(unsigned int a, int b) { return a > (unsigned int)b ? a : (unsigned int)b; }
inline unsigned int min(unsigned int a, int b) { return a < (unsigned int)b ? a : (unsigned int)b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline float max(float a, float b) { return a > b ? a : b; }
inline float min(float a, float b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
#endif
