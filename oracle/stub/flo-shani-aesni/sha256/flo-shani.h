/* Declaration-only stand-in for the flo-shani-aesni submodule header, which is
 * absent from the reference checkout.  The reference includes it from
 * include/infrastructure/my_hhash.h:9 but, with USESHA3 defined there, never
 * calls the SHA-256 routine, so a declaration is all the oracle build needs.
 * Test infrastructure only. */
#pragma once
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
void sha256_update_shani(const unsigned char *msg, size_t len, unsigned char *digest);
#ifdef __cplusplus
}
#endif
