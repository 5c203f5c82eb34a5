/* Build shim (test infrastructure only): QuRT threads, mutexes and condition
 * variables over POSIX threads (oracle/shim/shim.c). */
#ifndef ROVER_SHIM_QURT_H
#define ROVER_SHIM_QURT_H
#include <pthread.h>
#include <stdint.h>
#define QURT_EOK 0
#define QURT_EFAILED 12
#define QURT_THREAD_ATTR_NAME_MAXLEN 16
#define QURT_THREAD_ATTR_PRIORITY_DEFAULT 255
typedef pthread_t qurt_thread_t;
typedef struct { char name[QURT_THREAD_ATTR_NAME_MAXLEN]; unsigned int stack_size;
                 void *stack_addr; unsigned short priority; } qurt_thread_attr_t;
typedef pthread_mutex_t qurt_mutex_t;
typedef pthread_cond_t qurt_cond_t;
void qurt_thread_attr_init(qurt_thread_attr_t *attr);
void qurt_thread_attr_set_name(qurt_thread_attr_t *attr, const char *name);
void qurt_thread_attr_set_stack_size(qurt_thread_attr_t *attr, unsigned int size);
void qurt_thread_attr_set_stack_addr(qurt_thread_attr_t *attr, void *addr);
void qurt_thread_attr_set_priority(qurt_thread_attr_t *attr, unsigned short prio);
int qurt_thread_create(qurt_thread_t *thread, qurt_thread_attr_t *attr,
                       void (*entry)(void *), void *arg);
int qurt_thread_join(qurt_thread_t thread, int *status);
void qurt_thread_exit(int status);
void qurt_mutex_init(qurt_mutex_t *m);
void qurt_mutex_destroy(qurt_mutex_t *m);
void qurt_mutex_lock(qurt_mutex_t *m);
void qurt_mutex_unlock(qurt_mutex_t *m);
void qurt_cond_init(qurt_cond_t *c);
void qurt_cond_destroy(qurt_cond_t *c);
void qurt_cond_signal(qurt_cond_t *c);
void qurt_cond_broadcast(qurt_cond_t *c);
void qurt_cond_wait(qurt_cond_t *c, qurt_mutex_t *m);
#endif
