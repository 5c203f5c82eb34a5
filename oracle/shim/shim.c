/*
 * Host shim for building the reference Rover sources on x86-64 -- test
 * infrastructure for the oracle only; no search arithmetic lives here.
 *
 * It provides the platform calls the reference's DSP skeleton and host
 * pipeline make (QuRT threads, HAP mmap/perf/VTCM, rpcmem, fastrpc) so that
 * the unmodified reference code (src/app/dsp.c and the src/dsp_demo sources) links into
 * one in-process library.  rpcmem buffers are heap allocations named by
 * small integer "fds"; HAP_mmap_get resolves an fd to the same pointer, which
 * is what FastRPC's shared ION buffers give the DSP on the phone.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <pthread.h>
#include <sched.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "AEEStdDef.h"
#include "HAP_compute_res.h"
#include "HAP_mem.h"
#include "HAP_perf.h"
#include "qurt.h"
#include "qurt_memory.h"
#include "qurt_timer.h"
#include "remote.h"
#include "rpcmem.h"

#define SHIM_MAX_BUFFERS 4096
#define SHIM_FD_BASE 1000

typedef struct { void *ptr; size_t size; int live; } ShimBuffer;
static ShimBuffer g_buffers[SHIM_MAX_BUFFERS];
static pthread_mutex_t g_buffers_lock = PTHREAD_MUTEX_INITIALIZER;

void rpcmem_init(void) {}
void rpcmem_deinit(void) {}

void *rpcmem_alloc(int heapid, uint32_t flags, int size) {
    (void)heapid; (void)flags;
    if (size <= 0) return NULL;
    void *p = NULL;
    if (posix_memalign(&p, 4096, (size_t)size) != 0) return NULL;
    pthread_mutex_lock(&g_buffers_lock);
    for (int i = 0; i < SHIM_MAX_BUFFERS; i++) {
        if (!g_buffers[i].live) {
            g_buffers[i].ptr = p; g_buffers[i].size = (size_t)size; g_buffers[i].live = 1;
            pthread_mutex_unlock(&g_buffers_lock);
            return p;
        }
    }
    pthread_mutex_unlock(&g_buffers_lock);
    free(p);
    return NULL;
}

void rpcmem_free(void *po) {
    if (!po) return;
    pthread_mutex_lock(&g_buffers_lock);
    for (int i = 0; i < SHIM_MAX_BUFFERS; i++) {
        if (g_buffers[i].live && g_buffers[i].ptr == po) {
            g_buffers[i].live = 0; g_buffers[i].ptr = NULL;
            break;
        }
    }
    pthread_mutex_unlock(&g_buffers_lock);
    free(po);
}

int rpcmem_to_fd(void *po) {
    int fd = -1;
    pthread_mutex_lock(&g_buffers_lock);
    for (int i = 0; i < SHIM_MAX_BUFFERS; i++)
        if (g_buffers[i].live && g_buffers[i].ptr == po) { fd = SHIM_FD_BASE + i; break; }
    pthread_mutex_unlock(&g_buffers_lock);
    return fd;
}

int HAP_mmap_get(int fd, void **vaddr, uint64 *paddr) {
    int i = fd - SHIM_FD_BASE, rc = -1;
    pthread_mutex_lock(&g_buffers_lock);
    if (i >= 0 && i < SHIM_MAX_BUFFERS && g_buffers[i].live) {
        if (vaddr) *vaddr = g_buffers[i].ptr;
        if (paddr) *paddr = (uint64)(uintptr_t)g_buffers[i].ptr;
        rc = 0;
    }
    pthread_mutex_unlock(&g_buffers_lock);
    return rc;
}

int HAP_mmap_put(int fd) { (void)fd; return 0; }

int fastrpc_mmap(int domain, int fd, void *addr, int offset, size_t length,
                 enum fastrpc_map_flags flags) {
    (void)domain; (void)offset; (void)length; (void)flags;
    void *mapped = NULL;
    if (HAP_mmap_get(fd, &mapped, NULL) != 0 || mapped != addr) return -1;
    return 0;
}

int fastrpc_munmap(int domain, int fd, void *addr, size_t length) {
    (void)domain; (void)fd; (void)addr; (void)length;
    return 0;
}

int remote_session_control(uint32_t req, void *data, uint32_t datalen) {
    (void)req; (void)data; (void)datalen;
    return 0;
}

uint64_t HAP_perf_get_time_us(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (uint64_t)ts.tv_sec * 1000000ull + (uint64_t)ts.tv_nsec / 1000ull;
}

int HAP_compute_res_attr_init(compute_res_attr_t *attr) {
    if (attr) memset(attr, 0, sizeof(*attr));
    return 0;
}
int HAP_compute_res_attr_set_vtcm_param(compute_res_attr_t *attr, unsigned int size,
                                        unsigned int single_page) {
    (void)attr; (void)size; (void)single_page;
    return 0;
}
unsigned int HAP_compute_res_acquire(compute_res_attr_t *attr, unsigned int timeout_us) {
    (void)attr; (void)timeout_us;
    return 0; /* no VTCM on the host: context id 0 means "not granted" */
}
void *HAP_compute_res_attr_get_vtcm_ptr(compute_res_attr_t *attr) { (void)attr; return NULL; }
int HAP_compute_res_release(unsigned int context_id) { (void)context_id; return 0; }

int qurt_mem_cache_clean(qurt_addr_t addr, qurt_size_t size, qurt_mem_cache_op_t op,
                         qurt_mem_cache_type_t type) {
    (void)addr; (void)size; (void)op; (void)type;
    __sync_synchronize();
    return 0;
}

int qurt_timer_sleep(unsigned long long duration_us) {
    struct timespec ts = { (time_t)(duration_us / 1000000ull),
                           (long)(duration_us % 1000000ull) * 1000L };
    nanosleep(&ts, NULL);
    return QURT_EOK;
}

void qurt_thread_attr_init(qurt_thread_attr_t *attr) { if (attr) memset(attr, 0, sizeof(*attr)); }
void qurt_thread_attr_set_name(qurt_thread_attr_t *attr, const char *name) {
    if (attr && name) { strncpy(attr->name, name, sizeof(attr->name) - 1); }
}
void qurt_thread_attr_set_stack_size(qurt_thread_attr_t *attr, unsigned int size) {
    if (attr) attr->stack_size = size;
}
void qurt_thread_attr_set_stack_addr(qurt_thread_attr_t *attr, void *addr) {
    if (attr) attr->stack_addr = addr;
}
void qurt_thread_attr_set_priority(qurt_thread_attr_t *attr, unsigned short prio) {
    if (attr) attr->priority = prio;
}

typedef struct { void (*entry)(void *); void *arg; } ShimThreadStart;

static void *shim_thread_main(void *p) {
    ShimThreadStart start = *(ShimThreadStart *)p;
    free(p);
    start.entry(start.arg);
    return (void *)(intptr_t)QURT_EOK;
}

/* The reference hands QuRT a 4 KiB caller-owned stack; a host pthread gets
 * its own default-size stack instead. */
int qurt_thread_create(qurt_thread_t *thread, qurt_thread_attr_t *attr,
                       void (*entry)(void *), void *arg) {
    (void)attr;
    ShimThreadStart *start = (ShimThreadStart *)malloc(sizeof(*start));
    if (!start) return QURT_EFAILED;
    start->entry = entry; start->arg = arg;
    if (pthread_create(thread, NULL, shim_thread_main, start) != 0) {
        free(start);
        return QURT_EFAILED;
    }
    return QURT_EOK;
}

int qurt_thread_join(qurt_thread_t thread, int *status) {
    void *ret = NULL;
    int rc = pthread_join(thread, &ret);
    if (status) *status = (int)(intptr_t)ret;
    return rc == 0 ? QURT_EOK : QURT_EFAILED;
}

void qurt_thread_exit(int status) { pthread_exit((void *)(intptr_t)status); }

void qurt_mutex_init(qurt_mutex_t *m) { pthread_mutex_init(m, NULL); }
void qurt_mutex_destroy(qurt_mutex_t *m) { pthread_mutex_destroy(m); }
void qurt_mutex_lock(qurt_mutex_t *m) { pthread_mutex_lock(m); }
void qurt_mutex_unlock(qurt_mutex_t *m) { pthread_mutex_unlock(m); }
void qurt_cond_init(qurt_cond_t *c) { pthread_cond_init(c, NULL); }
void qurt_cond_destroy(qurt_cond_t *c) { pthread_cond_destroy(c); }
void qurt_cond_signal(qurt_cond_t *c) { pthread_cond_signal(c); }
void qurt_cond_broadcast(qurt_cond_t *c) { pthread_cond_broadcast(c); }
void qurt_cond_wait(qurt_cond_t *c, qurt_mutex_t *m) { pthread_cond_wait(c, m); }
