/* Host stand-in for <Windows.h> (reference-pinning harness): the reference's
 * device sources use nothing from it; its Win32 calls live in the host
 * program (INI parsing, file paths), which the harness does not compile. */
#ifndef GEGS_REF_SHIM_WINDOWS_H
#define GEGS_REF_SHIM_WINDOWS_H
#include <cstdio>
/* the one Win32 CRT call of the host set-up routines (init.cu:1168) */
static inline int fopen_s(FILE **f, const char *name, const char *mode)
{
    *f = std::fopen(name, mode);
    return *f ? 0 : 1;
}
#endif
