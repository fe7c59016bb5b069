/* Host stand-in for <Windows.h> (reference-pinning harness): the reference's
 * device sources use nothing from it; its Win32 calls live in the host
 * program (INI parsing, file paths), which the harness does not compile. */
#ifndef GEGS_REF_SHIM_WINDOWS_H
#define GEGS_REF_SHIM_WINDOWS_H
#endif
