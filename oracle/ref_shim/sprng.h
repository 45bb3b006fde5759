/* sprng.h -- TEST INFRASTRUCTURE ONLY.  Stand-in for SPRNG's simple interface
 * (sprng() returns the next uniform of this process's stream), the only SPRNG
 * call the reference makes (parallel_random_numbers.cpp:12-13).  The stream is
 * the oracle's Philox4x32-10 uniform stream (oracle/philox.h) keyed by a seed
 * and a stream number, so the reference's own polar method draws the same
 * normals the oracle draws; ref_sprng_reset() (re)starts it.  Declared with C
 * linkage (the reference includes this header inside extern "C"). */
#ifndef REF_SHIM_SPRNG_H
#define REF_SHIM_SPRNG_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
double sprng(void);
void ref_sprng_reset(uint64_t seed, uint64_t stream);
#ifdef __cplusplus
}
#endif
#endif
