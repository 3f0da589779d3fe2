/* oracle/shim/sep_stub.c -- aborting stand-ins for the SEPlib I/O entry points
 * the reference's IO.hpp templates reference (putch, auxputch, srite_big,
 * sreed_big, ...).  TEST INFRASTRUCTURE ONLY: the oracle drives the solver
 * with output "none", so none of these runs; reaching one is a bug. */
#include <stdio.h>
#include <stdlib.h>

static void sep_abort(const char *name)
{
    fprintf(stderr, "oracle: SEPlib routine %s is not available\n", name);
    abort();
}
int putch(char *a, char *b, void *c) { (void)a; (void)b; (void)c; sep_abort("putch"); return -1; }
int auxputch(const char *a, const char *b, const void *c, const char *d)
{
    (void)a; (void)b; (void)c; (void)d;
    sep_abort("auxputch");
    return -1;
}
size_t srite_big(const char *a, void *b, size_t c) { (void)a; (void)b; (void)c; sep_abort("srite_big"); return 0; }
size_t sreed_big(const char *a, void *b, size_t c) { (void)a; (void)b; (void)c; sep_abort("sreed_big"); return 0; }
