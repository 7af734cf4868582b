/* time_shim.c -- LD_PRELOAD shim that pins time(NULL) for the reference build.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference seeds its XORWOW generator with
 * time(NULL) (transport.cu:72) and has no seed option.  With
 * MCML_FIXED_TIME=<n> in the environment this shim makes time() return n,
 * which fixes the reference's seed without editing its sources.  Without
 * the variable it forwards to the C library's time().
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdlib.h>
#include <time.h>

time_t time(time_t *t) {
  const char *s = getenv("MCML_FIXED_TIME");
  time_t v;
  if (s) {
    v = (time_t)strtoll(s, NULL, 10);
  } else {
    time_t (*real)(time_t *) = (time_t(*)(time_t *))dlsym(RTLD_NEXT, "time");
    v = real ? real(NULL) : (time_t)0;
  }
  if (t) *t = v;
  return v;
}
