/* Test support, loaded with LD_PRELOAD into a child process of
 * tests/test_zz_no_alloc.py: counts the CUDA runtime calls that allocate or
 * free device or pinned host memory, then forwards each to libcudart.
 * oks_alloc_probe_reset() zeroes the count, oks_alloc_probe_count() reads it.
 * Build: gcc -shared -fPIC -O2 alloc_counter.c -o alloc_counter.so -ldl */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stddef.h>

static volatile long g_count = 0;

void oks_alloc_probe_reset(void) { g_count = 0; }
long oks_alloc_probe_count(void) { return g_count; }

typedef int (*fn2_t)(void*, size_t);
typedef int (*fn3_t)(void*, size_t, void*);
typedef int (*fn1_t)(void*);
typedef int (*fnf2_t)(void*, void*);
typedef int (*fnhost_t)(void*, size_t, unsigned int);
typedef int (*fnpitch_t)(void*, size_t*, size_t, size_t);
typedef int (*fnpool_t)(void*, size_t, void*, void*);

/* The real function: next in the global scope, else libcudart's own
 * definition (a library loaded with RTLD_LOCAL, e.g. through ctypes, keeps
 * libcudart out of the global scope). */
static void* real_fn(const char* name) {
    void* f = dlsym(RTLD_NEXT, name);
    if (!f) {
        void* h = dlopen("libcudart.so.12", RTLD_NOW | RTLD_NOLOAD);
        if (h) f = dlsym(h, name);
    }
    return f;
}
static int missing(void) { return 999; /* cudaErrorUnknown */ }
#define NEXT(type, name) (real_fn(name) ? (type)real_fn(name) : (type)missing)

int cudaMalloc(void* p, size_t n) { ++g_count; return NEXT(fn2_t, "cudaMalloc")(p, n); }
int cudaMallocHost(void* p, size_t n) { ++g_count; return NEXT(fn2_t, "cudaMallocHost")(p, n); }
int cudaMallocAsync(void* p, size_t n, void* s) { ++g_count; return NEXT(fn3_t, "cudaMallocAsync")(p, n, s); }
int cudaMallocManaged(void* p, size_t n, unsigned int f) {
    ++g_count;
    return NEXT(fnhost_t, "cudaMallocManaged")(p, n, f);
}
int cudaHostAlloc(void* p, size_t n, unsigned int f) { ++g_count; return NEXT(fnhost_t, "cudaHostAlloc")(p, n, f); }
int cudaMallocPitch(void* p, size_t* pitch, size_t w, size_t h) {
    ++g_count;
    return NEXT(fnpitch_t, "cudaMallocPitch")(p, pitch, w, h);
}
int cudaMallocFromPoolAsync(void* p, size_t n, void* pool, void* s) {
    ++g_count;
    return NEXT(fnpool_t, "cudaMallocFromPoolAsync")(p, n, pool, s);
}
int cudaFree(void* p) { ++g_count; return NEXT(fn1_t, "cudaFree")(p); }
int cudaFreeHost(void* p) { ++g_count; return NEXT(fn1_t, "cudaFreeHost")(p); }
int cudaFreeAsync(void* p, void* s) { ++g_count; return NEXT(fnf2_t, "cudaFreeAsync")(p, s); }
