/* Build shim (test infrastructure only): VTCM is never granted on the host,
 * so the reference takes its scalar ADC path. */
#ifndef ROVER_SHIM_HAP_COMPUTE_RES_H
#define ROVER_SHIM_HAP_COMPUTE_RES_H
typedef struct { unsigned long long opaque[8]; } compute_res_attr_t;
int HAP_compute_res_attr_init(compute_res_attr_t *attr);
int HAP_compute_res_attr_set_vtcm_param(compute_res_attr_t *attr,
                                        unsigned int size, unsigned int single_page);
unsigned int HAP_compute_res_acquire(compute_res_attr_t *attr, unsigned int timeout_us);
void *HAP_compute_res_attr_get_vtcm_ptr(compute_res_attr_t *attr);
int HAP_compute_res_release(unsigned int context_id);
#endif
