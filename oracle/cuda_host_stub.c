/*
 * cuda_host_stub.c -- host-memory stand-in for the CUDA runtime calls the
 * GOWalker headers make, so their CPU step can run on a machine without a GPU.
 *
 * TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libref_step*.so, the
 * harness that drives the reference's own sidewalkupdate.  Device allocations
 * become zeroed host allocations, copies become memcpy, kernel launches do
 * nothing (the harness never needs a kernel's result), streams are dummies.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int cudaError_t;
typedef void *cudaStream_t;
typedef struct { unsigned x, y, z; } stub_dim3;

cudaError_t cudaMalloc(void **p, size_t n) { *p = calloc(1, n ? n : 1); return *p ? 0 : 2; }
cudaError_t cudaMallocAsync(void **p, size_t n, cudaStream_t s) { (void)s; return cudaMalloc(p, n); }
cudaError_t cudaHostAlloc(void **p, size_t n, unsigned f) { (void)f; return cudaMalloc(p, n); }
cudaError_t cudaFree(void *p) { free(p); return 0; }
cudaError_t cudaFreeAsync(void *p, cudaStream_t s) { (void)s; free(p); return 0; }
cudaError_t cudaFreeHost(void *p) { free(p); return 0; }
cudaError_t cudaHostRegister(void *p, size_t n, unsigned f) { (void)p; (void)n; (void)f; return 0; }
cudaError_t cudaMemcpy(void *d, const void *s, size_t n, int k) { (void)k; if (n) memmove(d, s, n); return 0; }
cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n, int k, cudaStream_t st)
{
    (void)st;
    return cudaMemcpy(d, s, n, k);
}
cudaError_t cudaMemset(void *d, int v, size_t n) { memset(d, v, n); return 0; }
cudaError_t cudaMemsetAsync(void *d, int v, size_t n, cudaStream_t s) { (void)s; memset(d, v, n); return 0; }
cudaError_t cudaStreamCreate(cudaStream_t *s) { static int dummy; *s = &dummy; return 0; }
cudaError_t cudaStreamSynchronize(cudaStream_t s) { (void)s; return 0; }
cudaError_t cudaDeviceSynchronize(void) { return 0; }
cudaError_t cudaGetDeviceCount(int *n) { *n = 1; return 0; }
cudaError_t cudaSetDevice(int d) { (void)d; return 0; }
cudaError_t cudaGetLastError(void) { return 0; }
const char *cudaGetErrorString(cudaError_t e) { (void)e; return "stub"; }

cudaError_t cudaLaunchKernel(const void *f, stub_dim3 g, stub_dim3 b, void **a, size_t sm, cudaStream_t s)
{
    (void)f; (void)g; (void)b; (void)a; (void)sm; (void)s;
    return 0;
}

/* Registration hooks emitted by nvcc for the translation unit's kernels. */
void **__cudaRegisterFatBinary(void *fb) { static void *h[4]; (void)fb; return h; }
void __cudaRegisterFatBinaryEnd(void **h) { (void)h; }
void __cudaUnregisterFatBinary(void **h) { (void)h; }
void __cudaRegisterFunction(void **h, const char *hf, char *df, const char *dn, int tl, void *tid,
                            void *bid, void *bd, void *gd, int *ws)
{
    (void)h; (void)hf; (void)df; (void)dn; (void)tl; (void)tid; (void)bid; (void)bd; (void)gd; (void)ws;
}
void __cudaRegisterVar(void **h, char *hv, char *dh, const char *dn, int ext, size_t sz, int cst, int gl)
{
    (void)h; (void)hv; (void)dh; (void)dn; (void)ext; (void)sz; (void)cst; (void)gl;
}
void __cudaRegisterManagedVar(void **h, void **hv, char *dh, const char *dn, int ext, size_t sz, int cst,
                              int gl)
{
    (void)h; (void)hv; (void)dh; (void)dn; (void)ext; (void)sz; (void)cst; (void)gl;
}
char __cudaInitModule(void **h) { (void)h; return 0; }
unsigned __cudaPushCallConfiguration(stub_dim3 g, stub_dim3 b, size_t sm, void *s)
{
    (void)g; (void)b; (void)sm; (void)s;
    return 0;
}
cudaError_t __cudaPopCallConfiguration(stub_dim3 *g, stub_dim3 *b, size_t *sm, void *s)
{
    (void)g; (void)b; (void)sm; (void)s;
    return 0;
}
