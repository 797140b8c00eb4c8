/* c_caller.c -- a plain C caller of the drop-in interface, written the way the reference's
 * own callers use src/fast_mul.h (bench/bench.c:32-43,86: malloc'd limb buffers, one
 * abs_mul64 call, no other API): it includes include/fast_mul.h, links against
 * libfastmul_b200.so and nothing else, and reads/writes raw little-endian u64 files.
 *
 *   c_caller mul <in1.bin> <in2.bin> <out.bin>     out = in1 * in2
 *   c_caller sqr <in1.bin> <out.bin>               out = in1 * in1
 *   c_caller alias <in1.bin> <in2.bin> <out.bin>   the same product written over in1's
 *                                                   buffer (out may alias an input)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fast_mul.h"

static u64* read_limbs(const char* path, u64* n, u64 extra) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror(path);
        exit(2);
    }
    fseek(f, 0, SEEK_END);
    const long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    *n = (u64)bytes / sizeof(u64);
    u64* p = (u64*)malloc((size_t)(*n + extra) * sizeof(u64) + 8);
    if (!p || fread(p, sizeof(u64), (size_t)*n, f) != (size_t)*n) {
        fprintf(stderr, "reading %s failed\n", path);
        exit(2);
    }
    fclose(f);
    return p;
}

static void write_limbs(const char* path, const u64* p, u64 n) {
    FILE* f = fopen(path, "wb");
    if (!f || fwrite(p, sizeof(u64), (size_t)n, f) != (size_t)n) {
        fprintf(stderr, "writing %s failed\n", path);
        exit(2);
    }
    fclose(f);
}

int main(int argc, char** argv) {
    if (argc == 4 && strcmp(argv[1], "sqr") == 0) {
        u64 n;
        u64* a = read_limbs(argv[2], &n, 0);
        u64* out = (u64*)malloc((size_t)(2 * n) * sizeof(u64) + 8);
        abs_sqr64(a, n, out);
        write_limbs(argv[3], out, 2 * n);
        free(a);
        free(out);
        return 0;
    }
    if (argc == 5 && (strcmp(argv[1], "mul") == 0 || strcmp(argv[1], "alias") == 0)) {
        u64 n1, n2;
        const int alias = strcmp(argv[1], "alias") == 0;
        u64* a = read_limbs(argv[2], &n1, 0);
        u64* b = read_limbs(argv[3], &n2, 0);
        if (alias) {
            /* in1 sits at the start of a buffer long enough for the product */
            u64* big = (u64*)malloc((size_t)(n1 + n2) * sizeof(u64) + 8);
            memcpy(big, a, (size_t)n1 * sizeof(u64));
            abs_mul64(big, n1, b, n2, big);
            write_limbs(argv[4], big, n1 + n2);
            free(big);
        } else {
            u64* out = (u64*)malloc((size_t)(n1 + n2) * sizeof(u64) + 8);
            abs_mul64(a, n1, b, n2, out);
            write_limbs(argv[4], out, n1 + n2);
            free(out);
        }
        free(a);
        free(b);
        return 0;
    }
    fprintf(stderr, "usage: %s mul|alias <in1> <in2> <out> | sqr <in1> <out>\n", argv[0]);
    return 2;
}
