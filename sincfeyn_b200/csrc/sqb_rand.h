/* sqb_rand.h -- the C library's rand() stream after srand(seed), per caller.  glibc's rand() is random()
 * on its default 128-byte state (the additive feedback generator of TYPE_3); initstate_r()/random_r()
 * run the same generator on a private state, so concurrent callers do not share the process-wide one.
 * The reference draws its random nodes this way (driver/sum.c:468, 528; driver/main.c:80-81). */
#pragma once
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

struct SqbRand {
    random_data rd; char st[128];
    explicit SqbRand(unsigned seed){ memset(&rd, 0, sizeof rd); memset(st, 0, sizeof st); initstate_r(seed, st, sizeof st, &rd); }
    int next(){ int32_t r = 0; random_r(&rd, &r); return (int)r; }
};
