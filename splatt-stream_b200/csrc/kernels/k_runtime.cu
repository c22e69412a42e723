/*
 * k_runtime.cu -- device selection, stream, allocation, copies, events.
 */
#include "common.cuh"
#include "kstream.h"
#include <stdio.h>

namespace sb {

static cudaStream_t g_stream = nullptr;
static bool g_init = false;
static cudaError_t g_last = cudaSuccess;

cudaStream_t stream() { return g_stream; }

int fail(cudaError_t e)
{
  g_last = e;
  /* clear the sticky-free error so later calls are not poisoned */
  cudaGetLastError();
  if(e == cudaErrorMemoryAllocation) { return SB_ENOMEM; }
  return SB_EDEVICE;
}

} /* namespace sb */

using namespace sb;

extern "C" {

int sb_init(int device)
{
  if(g_init) { return SB_OK; }
  int n = 0;
  SB_TRY(cudaGetDeviceCount(&n));
  if(n == 0) { return fail(cudaErrorNoDevice); }
  if(device >= 0) { SB_TRY(cudaSetDevice(device)); }
  SB_TRY(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  /* keep freed stream-ordered memory in the pool rather than returning it */
  int dev = 0;
  SB_TRY(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  if(cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thresh = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh);
  }
  g_init = true;
  return SB_OK;
}

void * sb_get_stream(void) { return (void *) g_stream; }
void sb_set_stream(void * s) { g_stream = (cudaStream_t) s; }

int sb_sync(void)
{
  SB_TRY(cudaStreamSynchronize(g_stream));
  return SB_OK;
}

int sb_stream_sync(void * s)
{
  SB_TRY(cudaStreamSynchronize((cudaStream_t) s));
  return SB_OK;
}

int sb_malloc(void ** p, size_t bytes)
{
  if(bytes == 0) { bytes = 16; }
  SB_TRY(cudaMallocAsync(p, bytes, g_stream));
  return SB_OK;
}

int sb_free(void * p)
{
  if(p) { SB_TRY(cudaFreeAsync(p, g_stream)); }
  return SB_OK;
}

int sb_memset(void * p, int v, size_t bytes)
{
  if(bytes) { SB_TRY(cudaMemsetAsync(p, v, bytes, g_stream)); }
  return SB_OK;
}

int sb_h2d(void * dst, void const * src, size_t bytes)
{
  if(bytes) { SB_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g_stream)); }
  return SB_OK;
}

int sb_d2h(void * dst, void const * src, size_t bytes)
{
  if(bytes) {
    SB_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, g_stream));
    SB_TRY(cudaStreamSynchronize(g_stream));
  }
  return SB_OK;
}

int sb_d2d(void * dst, void const * src, size_t bytes)
{
  if(bytes) { SB_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, g_stream)); }
  return SB_OK;
}

/* ---- capture of a stream-ordered sequence into a CUDA graph ---- */
int sb_capture_begin(void)
{
  SB_TRY(cudaStreamBeginCapture(g_stream, cudaStreamCaptureModeThreadLocal));
  return SB_OK;
}

/* ends the capture; on success *exec is an instantiated graph.  A capture
 * that an unsupported call invalidated ends here with an error (and no
 * graph), leaving the stream usable. */
int sb_capture_end(void ** exec)
{
  *exec = nullptr;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(g_stream, &g);
  if(e != cudaSuccess || !g) {
    if(g) { cudaGraphDestroy(g); }
    return fail(e != cudaSuccess ? e : cudaErrorStreamCaptureInvalidated);
  }
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  if(e != cudaSuccess) { return fail(e); }
  *exec = (void *) x;
  return SB_OK;
}


int sb_host_alloc(void ** p, size_t bytes)
{
  SB_TRY(cudaHostAlloc(p, bytes ? bytes : 16, cudaHostAllocDefault));
  return SB_OK;
}

void sb_host_free(void * p)
{
  if(p) { cudaFreeHost(p); }
}

int sb_h2d_async(void * dst, void const * src, size_t bytes)
{
  if(bytes) { SB_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g_stream)); }
  return SB_OK;
}

/* 1 = the event has completed, 0 = not yet, < 0 = error */
int sb_event_query_done(void * ev)
{
  cudaError_t const e = cudaEventQuery((cudaEvent_t) ev);
  if(e == cudaSuccess) { return 1; }
  if(e == cudaErrorNotReady) { cudaGetLastError(); return 0; }
  fail(e);
  return -1;
}

int sb_graph_launch(void * g)
{
  SB_TRY(cudaGraphLaunch((cudaGraphExec_t) g, g_stream));
  return SB_OK;
}

void sb_graph_destroy(void * g)
{
  if(g) { cudaGraphExecDestroy((cudaGraphExec_t) g); }
}

int sb_last_error(void) { return (int) g_last; }
char const * sb_error_string(void) { return cudaGetErrorString(g_last); }

size_t sb_mem_free(void)
{
  size_t f = 0, t = 0;
  cudaMemGetInfo(&f, &t);
  return f;
}

int sb_device_count(void)
{
  int n = 0;
  if(cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int sb_event_create(void ** ev)
{
  SB_TRY(cudaEventCreate((cudaEvent_t *) ev));
  return SB_OK;
}

int sb_event_record(void * ev, void * s)
{
  SB_TRY(cudaEventRecord((cudaEvent_t) ev, s ? (cudaStream_t) s : g_stream));
  return SB_OK;
}

int sb_event_elapsed_ms(void * a, void * b, float * ms)
{
  SB_TRY(cudaEventSynchronize((cudaEvent_t) b));
  SB_TRY(cudaEventElapsedTime(ms, (cudaEvent_t) a, (cudaEvent_t) b));
  return SB_OK;
}

int sb_event_sync(void * ev)
{
  SB_TRY(cudaEventSynchronize((cudaEvent_t) ev));
  return SB_OK;
}

int sb_event_destroy(void * ev)
{
  SB_TRY(cudaEventDestroy((cudaEvent_t) ev));
  return SB_OK;
}

} /* extern "C" */
