/* Test infrastructure: force-included ahead of the reference's ray-tracing device source
 * when it is compiled for the host, so that its per-ray diagnostic printf (InnerRayTracing,
 * "undef inner trace") does not flood the test output. */
#include <cstdio>
static inline int rrhd_quiet_printf(const char *, ...) { return 0; }
#define printf rrhd_quiet_printf
