/*
 * TEST INFRASTRUCTURE ONLY — used to compile the reference's own sources into oracle/_ref/.
 *
 * Declaration-only stand-in for SpookyHash V2 (extlib/sux, empty in this checkout), which the
 * reference's util/Hash128.h names for string keys. The reference build in oracle/_ref/ is
 * driven with 128-bit keys only (string keys are hashed beforehand by this project's own
 * SpookyHash restatement), so calling this function is an error and aborts loudly.
 */
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>

class SpookyHash {
  public:
    static void Hash128(const void *, size_t, uint64_t *, uint64_t *) {
        std::fprintf(stderr, "oracle/_ref: string hashing is not part of the reference build; pass 128-bit keys\n");
        std::abort();
    }
};
