/*
 * mexhost.c -- a non-MATLAB host for MEX gateways.
 *
 * Implements the mxArray/MEX calls declared in matrix.h and mex.h so that a
 * gateway written for MATLAB (`void mexFunction(int, mxArray**, int,
 * const mxArray**)`) can be compiled with plain gcc and called from C or
 * Python (ctypes).  Semantics that the mela_* gateways depend on:
 *
 *   - mxCreateLogicalMatrix returns zero-filled storage (MATLAB does too).
 *   - mxCalloc(n, size) with n*size == 0 returns NULL.  The reference
 *     null-space gateways test the result of mxCalloc(m*wc) for NULL and
 *     report "Out of memory." when it is (mela_null_gf2.c:163-166 of the
 *     reference), so empty inputs reproduce that message here.
 *   - mexErrMsgTxt / mexErrMsgIdAndTxt long-jump back to mexhost_call(),
 *     which then frees every block still held from mxCalloc/mxMalloc.
 *   - allocation tracking is mutex-protected: the reference gateways call
 *     mxCalloc/mxFree from inside OpenMP parallel regions.
 */
#include "mex.h"

#include <pthread.h>
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct block_tag {
    struct block_tag *prev, *next;
    /* payload follows, 64-byte aligned */
} block_t;

#define BLOCK_HDR 64

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static block_t g_head = {&g_head, &g_head};

static __thread jmp_buf *t_jmp = NULL;
static __thread char t_err_id[256];
static __thread char t_err_msg[1024];

static void *track_alloc(size_t bytes, int zero)
{
    unsigned char *raw = (unsigned char *)malloc(bytes + BLOCK_HDR);
    if (!raw) return NULL;
    if (zero) memset(raw + BLOCK_HDR, 0, bytes);
    block_t *b = (block_t *)raw;
    pthread_mutex_lock(&g_lock);
    b->next = g_head.next;
    b->prev = &g_head;
    g_head.next->prev = b;
    g_head.next = b;
    pthread_mutex_unlock(&g_lock);
    return raw + BLOCK_HDR;
}

void *mxCalloc(size_t n, size_t size)
{
    if (n == 0 || size == 0) return NULL;
    if (size != 0 && n > ((size_t)-1 - BLOCK_HDR) / size) return NULL;
    return track_alloc(n * size, 1);
}

void *mxMalloc(size_t n)
{
    if (n == 0) return NULL;
    return track_alloc(n, 0);
}

void mxFree(void *p)
{
    if (!p) return;
    block_t *b = (block_t *)((unsigned char *)p - BLOCK_HDR);
    pthread_mutex_lock(&g_lock);
    b->prev->next = b->next;
    b->next->prev = b->prev;
    pthread_mutex_unlock(&g_lock);
    free(b);
}

static void free_all_tracked(void)
{
    pthread_mutex_lock(&g_lock);
    block_t *b = g_head.next;
    while (b != &g_head) {
        block_t *nx = b->next;
        free(b);
        b = nx;
    }
    g_head.next = g_head.prev = &g_head;
    pthread_mutex_unlock(&g_lock);
}

static size_t class_size(mxClassID c)
{
    switch (c) {
    case mxLOGICAL_CLASS: case mxINT8_CLASS: case mxUINT8_CLASS: case mxCHAR_CLASS: return 1;
    case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    default: return 1;
    }
}

mwSize mxGetM(const mxArray *a) { return a->m; }
mwSize mxGetN(const mxArray *a) { return a->n; }
bool mxIsDouble(const mxArray *a) { return a->classid == mxDOUBLE_CLASS; }
bool mxIsLogical(const mxArray *a) { return a->classid == mxLOGICAL_CLASS; }
bool mxIsSparse(const mxArray *a) { return a->sparse != 0; }
void *mxGetData(const mxArray *a) { return a->data; }
double *mxGetPr(const mxArray *a) { return (double *)a->data; }
mxLogical *mxGetLogicals(const mxArray *a) { return (mxLogical *)a->data; }
mxClassID mxGetClassID(const mxArray *a) { return a->classid; }

static mxArray *create(mxClassID cls, mwSize m, mwSize n)
{
    mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
    if (!a) return NULL;
    a->classid = cls;
    a->m = m;
    a->n = n;
    size_t bytes = m * n * class_size(cls);
    a->data = calloc(bytes ? bytes : 1, 1);
    a->owns_data = 1;
    if (!a->data) {
        free(a);
        return NULL;
    }
    return a;
}

mxArray *mxCreateLogicalMatrix(mwSize m, mwSize n) { return create(mxLOGICAL_CLASS, m, n); }

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c)
{
    (void)c; /* real storage only: the gateways create real outputs */
    return create(mxDOUBLE_CLASS, m, n);
}

mxArray *mxCreateDoubleScalar(double v)
{
    mxArray *a = create(mxDOUBLE_CLASS, 1, 1);
    if (a) ((double *)a->data)[0] = v;
    return a;
}

void mxDestroyArray(mxArray *a)
{
    if (!a) return;
    if (a->owns_data) free(a->data);
    free(a);
}

mxArray *mexhost_wrap(mxClassID cls, mwSize m, mwSize n, void *data, int sparse)
{
    mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
    if (!a) return NULL;
    a->classid = cls;
    a->m = m;
    a->n = n;
    a->data = data;
    a->sparse = sparse;
    a->owns_data = 0;
    return a;
}

void mexErrMsgTxt(const char *msg)
{
    t_err_id[0] = '\0';
    snprintf(t_err_msg, sizeof t_err_msg, "%s", msg ? msg : "");
    if (t_jmp) longjmp(*t_jmp, 1);
    fprintf(stderr, "mexErrMsgTxt outside mexhost_call: %s\n", t_err_msg);
    abort();
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...)
{
    snprintf(t_err_id, sizeof t_err_id, "%s", id ? id : "");
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err_msg, sizeof t_err_msg, fmt ? fmt : "", ap);
    va_end(ap);
    if (t_jmp) longjmp(*t_jmp, 1);
    fprintf(stderr, "mexErrMsgIdAndTxt outside mexhost_call: %s\n", t_err_msg);
    abort();
}

int mexPrintf(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int r = vprintf(fmt, ap);
    va_end(ap);
    return r;
}

int mexhost_call(mexhost_gateway_fn fn, int nlhs, mxArray *plhs[], int nrhs,
                 const mxArray *prhs[], char *err_id, size_t id_cap,
                 char *err_msg, size_t msg_cap)
{
    jmp_buf env;
    jmp_buf *saved = t_jmp;
    t_jmp = &env;
    if (setjmp(env) == 0) {
        fn(nlhs, plhs, nrhs, prhs);
        t_jmp = saved;
        free_all_tracked();
        return 0;
    }
    t_jmp = saved;
    free_all_tracked();
    for (int i = 0; i < nlhs; ++i) {
        /* outputs created before the error are discarded, as in MATLAB */
        if (plhs[i]) {
            mxDestroyArray(plhs[i]);
            plhs[i] = NULL;
        }
    }
    if (err_id && id_cap) snprintf(err_id, id_cap, "%s", t_err_id);
    if (err_msg && msg_cap) snprintf(err_msg, msg_cap, "%s", t_err_msg);
    return 1;
}
