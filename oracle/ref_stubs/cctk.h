/* Minimal stand-in for the Cactus flesh header, sufficient for compiling the
 * reference transfer operators (CarpetX/src/prolongate_3d_rf2*.cxx) outside
 * Cactus.  Test infrastructure only: this is part of the oracle build. */
#ifndef CX_REF_STUB_CCTK_H
#define CX_REF_STUB_CCTK_H
#include <cstdio>
#include <cstdlib>
typedef double CCTK_REAL;
typedef int CCTK_INT;
#define CCTK_DEVICE
#define CCTK_HOST
#define CCTK_ATTRIBUTE_NOINLINE __attribute__((__noinline__))
#define CCTK_ATTRIBUTE_ALWAYS_INLINE __attribute__((__always_inline__))
#define CCTK_BUILTIN_EXPECT(x, y) __builtin_expect(x, y)
#ifndef restrict
#define restrict __restrict__
#endif
#define CCTK_VERROR(...)                                                       \
  do {                                                                         \
    std::fprintf(stderr, __VA_ARGS__);                                         \
    std::fputc('\n', stderr);                                                  \
    std::abort();                                                              \
  } while (0)
#define CCTK_ERROR(msg) CCTK_VERROR("%s", msg)
#define CCTK_VINFO(...) ((void)0)
#define CCTK_VWARN(...) ((void)0)
#define CCTK_WARN(...) ((void)0)
#endif
