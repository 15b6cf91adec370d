/*
 * Test infrastructure only: lets the unchanged reference sources (an MSVC
 * project) compile with g++ on Linux so that its multi-domain TDBEM solver can
 * serve as the parity oracle.  Nothing here is part of the product library.
 *
 * Each definition maps one MSVC "secure CRT" or Win32 name used by the
 * reference onto its POSIX/C99 counterpart with the same observable behaviour
 * for the calls the reference makes.
 */
#ifndef TDBEM_ORACLE_WIN32_COMPAT_H
#define TDBEM_ORACLE_WIN32_COMPAT_H

#ifdef __cplusplus
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cerrno>
#else
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <errno.h>
#endif
#include <strings.h>
#include <unistd.h>
#include <sys/stat.h>
#include <sys/types.h>

typedef long long __int64;

static inline int fopen_s(FILE** fp, const char* name, const char* mode)
{
    *fp = fopen(name, mode);
    return *fp ? 0 : errno;
}

static inline int _dupenv_s(char** value, size_t* len, const char* name)
{
    const char* v = getenv(name);
    if (!v) {
        *value = 0;
        if (len) *len = 0;
        return 0;
    }
    *value = strdup(v);
    if (len) *len = strlen(v) + 1;
    return 0;
}

static inline char* _getcwd(char* buf, int size)
{
    return getcwd(buf, (size_t)size);
}

static inline int _mkdir(const char* path) { return mkdir(path, 0755); }
static inline int _finite(double v) { return __builtin_isfinite(v) ? 1 : 0; }
static inline int _strnicmp(const char* a, const char* b, size_t n) { return strncasecmp(a, b, n); }
static inline long long _ftelli64(FILE* f) { return (long long)ftello(f); }
static inline int _fseeki64(FILE* f, long long off, int whence) { return fseeko(f, (off_t)off, whence); }

static inline int _itoa_s(int value, char* buf, int radix)
{
    (void)radix;
    sprintf(buf, "%d", value);
    return 0;
}

#ifdef __cplusplus
/* sprintf_s comes in an array form (size deduced) and a pointer+size form. */
template <size_t N, typename... A>
static inline int sprintf_s(char (&dst)[N], const char* fmt, A... a) { return snprintf(dst, N, fmt, a...); }
template <typename... A>
static inline int sprintf_s(char* dst, size_t n, const char* fmt, A... a) { return snprintf(dst, n, fmt, a...); }
template <size_t N>
static inline int strcpy_s(char (&dst)[N], const char* src) { strncpy(dst, src, N - 1); dst[N - 1] = 0; return 0; }
template <size_t N>
static inline int strcat_s(char (&dst)[N], const char* src) { strncat(dst, src, N - strlen(dst) - 1); return 0; }
#endif
static inline int strcpy_s(char* dst, size_t n, const char* src) { strncpy(dst, src, n - 1); dst[n - 1] = 0; return 0; }
static inline int strcat_s(char* dst, size_t n, const char* src) { strncat(dst, src, n - strlen(dst) - 1); return 0; }

/* The secure scanf family takes an extra buffer-size argument after each %s
 * conversion; plain fscanf ignores surplus arguments, so the mapping is 1:1. */
#define printf_s printf
#define fprintf_s fprintf
#define scanf_s scanf
#define fscanf_s fscanf
#define _countof(a) (sizeof(a) / sizeof((a)[0]))

#endif
