/*
 * ref_prelude.h — force-included when compiling the reference's Tier-1 sources in place.
 * With no platform macro defined the reference selects its portable C++ Tier-1 path
 * (decoder/codec/include/codec.h:28-56: ENABLE_ASSEMBLY_OPTIMIZATION stays 0); its headers
 * then expect a few Windows-toolchain names, supplied here.  No reference source is copied.
 */
#include <string.h>
typedef void *HANDLE;
typedef unsigned long DWORD;
typedef long long _int64;
