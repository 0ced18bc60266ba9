/* Pipe runner over the plan API, speaking the wire protocol of the reference's runner
 * (tests/test_runner.c:19-52), so that drivers written for it (tests/verify_portability.py,
 * dataset/evaluate.py) run unchanged against this library.
 *
 * Each request is four little-endian uint32 {0x42524443, height, width, mode} followed by
 * height*width float32.  Each reply is four uint32 {magic, status of bridct_plan_apply, 1 if the
 * four guard floats on both sides of the input and output buffers are untouched, 1 if the input
 * is unchanged} followed by the output floats.  Exit codes: 0 at end of input, 2 malformed
 * request, 3 allocation or plan failure, 4 truncated payload, 5 write failure, 6 read error.
 *
 * Plans are kept while consecutive requests have the same shape (plan creation sets up device
 * staging); the results do not depend on it. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bridct.h"

#define RUNNER_MAGIC UINT32_C(0x42524443)
#define GUARD 4
static const float guard_value = 12345.0f;

static int guards_intact(const float *buf, size_t n)
{
    for (size_t i = 0; i < GUARD; ++i)
        if (buf[i] != guard_value || buf[GUARD + n + i] != guard_value)
            return 0;
    return 1;
}

int main(void)
{
    bridct_plan *plan = NULL;
    int plan_h = 0, plan_w = 0;
    size_t capacity = 0;
    float *in = NULL, *out = NULL, *copy = NULL;
    uint32_t head[4];
    size_t got;
    while ((got = fread(head, 1, sizeof head, stdin)) != 0) {
        if (got != sizeof head || head[0] != RUNNER_MAGIC || head[3] > 2 ||
            !bridct_supported((int)head[1], (int)head[2]))
            return 2;
        const int h = (int)head[1], w = (int)head[2];
        const size_t n = (size_t)h * (size_t)w;
        if (n > capacity) {
            free(in);
            free(out);
            free(copy);
            in = malloc((n + 2 * GUARD) * sizeof(float));
            out = malloc((n + 2 * GUARD) * sizeof(float));
            copy = malloc(n * sizeof(float));
            capacity = n;
            if (!in || !out || !copy)
                return 3;
        }
        if (!plan || plan_h != h || plan_w != w) {
            bridct_plan_destroy(plan);
            plan = bridct_plan_create(h, w);
            plan_h = h;
            plan_w = w;
            if (!plan)
                return 3;
        }
        for (size_t i = 0; i < n + 2 * GUARD; ++i)
            in[i] = out[i] = guard_value;
        if (fread(in + GUARD, sizeof(float), n, stdin) != n)
            return 4;
        memcpy(copy, in + GUARD, n * sizeof(float));
        const int status = bridct_plan_apply(plan, (enum bridct_mode)head[3], in + GUARD, out + GUARD);
        const uint32_t reply[4] = {head[0], (uint32_t)status,
                                   (uint32_t)(guards_intact(in, n) && guards_intact(out, n)),
                                   (uint32_t)(memcmp(copy, in + GUARD, n * sizeof(float)) == 0)};
        if (fwrite(reply, sizeof reply, 1, stdout) != 1 || fwrite(out + GUARD, sizeof(float), n, stdout) != n ||
            fflush(stdout) != 0)
            return 5;
    }
    bridct_plan_destroy(plan);
    free(in);
    free(out);
    free(copy);
    return ferror(stdin) ? 6 : 0;
}
