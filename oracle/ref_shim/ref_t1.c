/*
 * ref_t1.c -- host driver for the reference's Tier-1 kernel g_decode
 * (coefficient_coder.cl:778-819), compiled from the reference source with
 * cl_shim.h.  TEST INFRASTRUCTURE ONLY.
 *
 * The driver lays the blocks out as CoefficientCoder::decodeInit does
 * (CoefficientCoder.cpp:140-212): a 16 KiB codestream slot per block, a
 * state buffer of width*(stripes+2) words whose block pointer is offset by
 * one row, and a nominal-size output slot per block; then it runs one
 * work-item per block on a pool of host threads.
 */
#include "cl_shim.h"
#include "coefficient_coder.cl"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

__thread size_t shim_gid[3], shim_lid[3], shim_grp[3];

#define SLOT (4096 * 4) /* MAX_CODESTREAM_SIZE, CoefficientCoder.h:8 */

typedef struct {
    unsigned int *st;
    unsigned char *cs;
    CodeBlockAdditionalInfo *info;
    int n;
    int *out;
    int next;
} job_t;

static void *worker(void *p)
{
    job_t *J = (job_t *)p;
    for (;;) {
        const int i = __atomic_fetch_add(&J->next, 1, __ATOMIC_RELAXED);
        if (i >= J->n) break;
        shim_gid[0] = (size_t)i;
        g_decode(J->st, J->cs, SLOT, J->info, J->n, J->out);
    }
    return NULL;
}

/* Decode n blocks.  Per block: codeword, its length, width/height (<= 64),
 * orientation class (0 LL/LH, 1 HL, 2 HH), Mb and the number of coded
 * bit-planes (significant_bits).  out receives n slots of 64x64 int32 in the
 * reference's sign-magnitude format.  Returns the number of blocks skipped
 * because their codeword exceeds the 16 KiB slot. */
#ifndef REF_T1_NAME
#define REF_T1_NAME ref_t1_decode
#endif
int REF_T1_NAME(int n, const unsigned char *const *segs, const int *lens, const int *w, const int *h,
                const int *cls, const int *mb, const int *sigbits, int *out, int threads)
{
    CodeBlockAdditionalInfo *info = calloc((size_t)n, sizeof *info);
    unsigned char *cs = calloc((size_t)n, SLOT);
    size_t stn = 0;
    int skipped = 0;
    for (int i = 0; i < n; i++) stn += (size_t)w[i] * ((h[i] + 3) / 4 + 2);
    unsigned int *st = calloc(stn + 1, sizeof *st);
    size_t mo = 0;
    for (int i = 0; i < n; i++) {
        CodeBlockAdditionalInfo *b = &info[i];
        const int stripes = (h[i] + 3) / 4;
        b->width = (unsigned char)w[i];
        b->height = (unsigned char)h[i];
        b->nominalWidth = 64;
        b->nominalHeight = 64;
        b->stripeNo = (unsigned char)stripes;
        b->subband = (unsigned char)cls[i];
        b->magbits = (unsigned char)mb[i];
        b->significantBits = (unsigned char)sigbits[i];
        b->magconOffset = (int)(mo + (size_t)w[i]);
        b->d_coefficientsOffset = i * 64 * 64;
        if (lens[i] > SLOT) {
            b->length = 0;
            b->significantBits = 0;
            skipped++;
        } else {
            b->length = lens[i];
            memcpy(cs + (size_t)i * SLOT, segs[i], (size_t)lens[i]);
        }
        mo += (size_t)w[i] * (stripes + 2);
    }
    memset(out, 0, sizeof(int) * (size_t)n * 64 * 64);
    job_t J = {st, cs, info, n, out, 0};
    int nt = threads > 0 ? threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    pthread_t tid[256];
    if (nt > 256) nt = 256;
    if (nt > n) nt = n;
    int started = 0;
    for (int t = 0; t < nt; t++)
        if (!pthread_create(&tid[t], NULL, worker, &J)) started++;
    for (int t = 0; t < started; t++) pthread_join(tid[t], NULL);
    if (!started) worker(&J);
    free(info);
    free(cs);
    free(st);
    return skipped;
}
