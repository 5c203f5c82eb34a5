/* sha256.c -- SHA-256 (FIPS 180-4) for bundle member checks.
 *
 * Rover's index.json records a SHA-256 per member and the PQ / residual
 * headers carry one for their payloads (tools/index_bundle.py:187-226,
 * src/dsp_demo/retrieval_pq_artifact.c, retrieval_pq_residual.c:216-246).
 * The round constants are derived here from their definition -- the first
 * 32 bits of the fractional parts of the cube roots of the first 64 primes
 * (K) and of the square roots of the first 8 primes (initial H) -- with exact
 * integer roots, rather than tabulated. */
#define _FILE_OFFSET_BITS 64
#define _POSIX_C_SOURCE 200809L
#include "rover_host.h"

#include <stdio.h>
#include <sys/types.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static uint32_t K[64], H0[8];
static int ready = 0;

/* floor(x^(1/e)) for e = 2 or 3, exactly, by bisection */
static uint64_t iroot(u128 x, int e) {
    uint64_t lo = 0, hi = (uint64_t)1 << (e == 2 ? 40 : 36);
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo + 1) / 2;
        u128 p = (u128)mid * mid;
        if (e == 3) p *= mid;
        if (p <= x) lo = mid; else hi = mid - 1;
    }
    return lo;
}

static void init_constants(void) {
    int primes[64], count = 0;
    for (int c = 2; count < 64; ++c) {
        int prime = 1;
        for (int d = 2; d * d <= c; ++d)
            if (c % d == 0) { prime = 0; break; }
        if (prime) primes[count++] = c;
    }
    /* the fraction's first 32 bits = floor(root(p) * 2^32) mod 2^32 */
    for (int i = 0; i < 64; ++i) K[i] = (uint32_t)iroot((u128)primes[i] << 96, 3);
    for (int i = 0; i < 8; ++i) H0[i] = (uint32_t)iroot((u128)primes[i] << 64, 2);
    ready = 1;
}

static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

static void compress(uint32_t h[8], const uint8_t block[64]) {
    uint32_t w[64];
    for (int t = 0; t < 16; ++t)
        w[t] = (uint32_t)block[4 * t] << 24 | (uint32_t)block[4 * t + 1] << 16 | (uint32_t)block[4 * t + 2] << 8 |
               block[4 * t + 3];
    for (int t = 16; t < 64; ++t) {
        const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
        const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
        w[t] = w[t - 16] + s0 + w[t - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], k = h[7];
    for (int t = 0; t < 64; ++t) {
        const uint32_t t1 = k + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + K[t] + w[t];
        const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        k = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += k;
}

void rover_sha256_init(RoverSha256* s) {
    if (!ready) init_constants();
    memcpy(s->h, H0, sizeof(H0));
    s->bytes = 0;
    s->fill = 0;
}

void rover_sha256_update(RoverSha256* s, const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    s->bytes += len;
    if (s->fill) {
        const size_t take = len < 64 - s->fill ? len : 64 - s->fill;
        memcpy(s->buf + s->fill, p, take);
        s->fill += take;
        p += take;
        len -= take;
        if (s->fill < 64) return;
        compress(s->h, s->buf);
        s->fill = 0;
    }
    for (; len >= 64; p += 64, len -= 64) compress(s->h, p);
    memcpy(s->buf, p, len);
    s->fill = len;
}

void rover_sha256_final(RoverSha256* s, uint8_t out[32]) {
    const uint64_t bits = s->bytes * 8u;
    uint8_t pad[72] = {0x80};
    const size_t padlen = (s->fill < 56 ? 56 : 120) - s->fill;
    for (int i = 0; i < 8; ++i) pad[padlen + i] = (uint8_t)(bits >> (56 - 8 * i));
    rover_sha256_update(s, pad, padlen + 8);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(s->h[i] >> 24);
        out[4 * i + 1] = (uint8_t)(s->h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(s->h[i] >> 8);
        out[4 * i + 3] = (uint8_t)s->h[i];
    }
}

void rover_sha256(const void* data, size_t len, uint8_t out[32]) {
    RoverSha256 s;
    rover_sha256_init(&s);
    rover_sha256_update(&s, data, len);
    rover_sha256_final(&s, out);
}

int rover_sha256_file(const char* path, long long offset, uint8_t out[32]) {
    FILE* f = fopen(path, "rb");
    if (!f) return -1;
    if (offset > 0 && fseeko(f, (off_t)offset, SEEK_SET) != 0) {
        fclose(f);
        return -1;
    }
    const size_t chunk_bytes = (size_t)8 << 20;
    uint8_t* chunk = (uint8_t*)malloc(chunk_bytes);
    if (!chunk) {
        fclose(f);
        return -1;
    }
    RoverSha256 s;
    rover_sha256_init(&s);
    size_t got;
    while ((got = fread(chunk, 1, chunk_bytes, f)) > 0) rover_sha256_update(&s, chunk, got);
    const int bad = ferror(f);
    fclose(f);
    free(chunk);
    if (bad) return -1;
    rover_sha256_final(&s, out);
    return 0;
}

void rover_hex(const uint8_t* bytes, size_t len, char* out) {
    static const char digits[] = "0123456789abcdef";
    for (size_t i = 0; i < len; ++i) {
        out[2 * i] = digits[bytes[i] >> 4];
        out[2 * i + 1] = digits[bytes[i] & 15];
    }
    out[2 * len] = '\0';
}
