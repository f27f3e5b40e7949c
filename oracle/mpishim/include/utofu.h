/*
 * utofu.h stand-in for building the reference library off Fugaku (oracle
 * test infrastructure only).
 *
 * The reference compiles its uTofu transport (lib/fugaku/bine_utofu.cc) and
 * the uTofu members of BineCommon whenever FUGAKU is defined, and FUGAKU is
 * the only configuration in which its unguarded ring/bucket code compiles.
 * The oracle never selects the uTofu layer (every collective is forced onto
 * the MPI layer), so these declarations only have to let that code compile
 * and let BineCommon's constructor (lib/libbine_common.cc:159-176) run: the
 * set-up calls succeed, the data-path calls report an error.  Type and
 * function names follow the uTofu API as the reference uses it.
 */
#ifndef BINE_MPISHIM_UTOFU_H
#define BINE_MPISHIM_UTOFU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint64_t utofu_vcq_id_t;
typedef uint64_t utofu_stadd_t;
typedef void *utofu_vcq_hdl_t;
typedef int utofu_tni_id_t;
typedef uint64_t utofu_path_id_t;

struct utofu_mrq_notice {
    uint8_t notice_type;
    uint8_t padding1[3];
    uint32_t edata;
    utofu_vcq_id_t vcq_id;
    uint64_t rmt_value;
    utofu_stadd_t lcl_stadd;
    utofu_stadd_t rmt_stadd;
};

struct utofu_onesided_caps {
    uint64_t flags;
    size_t max_putget_size;
    size_t max_piggyback_size;
    size_t num_reserved_stags;
};

enum {
    UTOFU_SUCCESS = 0,
    UTOFU_ERR_NOT_FOUND = 1,
    UTOFU_ERR_BUSY = 2,
    UTOFU_ERR_NOT_SUPPORTED = 3,
    UTOFU_ERR_FATAL = 99
};

enum {
    UTOFU_MRQ_TYPE_LCL_PUT = 0,
    UTOFU_MRQ_TYPE_RMT_PUT = 1,
    UTOFU_MRQ_TYPE_LCL_GET = 2,
    UTOFU_MRQ_TYPE_RMT_GET = 3
};

#define UTOFU_ONESIDED_FLAG_TCQ_NOTICE        (1UL << 0)
#define UTOFU_ONESIDED_FLAG_REMOTE_MRQ_NOTICE (1UL << 1)
#define UTOFU_ONESIDED_FLAG_LOCAL_MRQ_NOTICE  (1UL << 2)
#define UTOFU_ONESIDED_FLAG_STRONG_ORDER      (1UL << 3)
#define UTOFU_ONESIDED_FLAG_DELAY_START       (1UL << 4)
#define UTOFU_VCQ_FLAG_EXCLUSIVE              (1UL << 0)
#define UTOFU_VCQ_FLAG_THREAD_SAFE            (1UL << 1)
#define UTOFU_THREAD_SAFE                     UTOFU_VCQ_FLAG_THREAD_SAFE

int utofu_get_onesided_tnis(utofu_tni_id_t **tni_ids, size_t *num_tnis);
int utofu_query_onesided_caps(utofu_tni_id_t tni_id, struct utofu_onesided_caps **caps);
int utofu_create_vcq(utofu_tni_id_t tni_id, unsigned long flags, utofu_vcq_hdl_t *vcq_hdl);
int utofu_free_vcq(utofu_vcq_hdl_t vcq_hdl);
int utofu_query_vcq_id(utofu_vcq_hdl_t vcq_hdl, utofu_vcq_id_t *vcq_id);
int utofu_set_vcq_id_path(utofu_vcq_id_t *vcq_id, uint8_t *path_coords);
int utofu_reg_mem(utofu_vcq_hdl_t vcq_hdl, void *addr, size_t size, unsigned long flags, utofu_stadd_t *stadd);
int utofu_dereg_mem(utofu_vcq_hdl_t vcq_hdl, utofu_stadd_t stadd, unsigned long flags);
int utofu_put(utofu_vcq_hdl_t vcq_hdl, utofu_vcq_id_t rmt_vcq_id, utofu_stadd_t lcl_stadd,
              utofu_stadd_t rmt_stadd, size_t length, uint64_t edata, unsigned long flags, void *cbvalue);
int utofu_put_piggyback(utofu_vcq_hdl_t vcq_hdl, utofu_vcq_id_t rmt_vcq_id, void *lcl_data,
                        utofu_stadd_t rmt_stadd, size_t length, uint64_t edata, unsigned long flags, void *cbvalue);
int utofu_poll_tcq(utofu_vcq_hdl_t vcq_hdl, unsigned long flags, void **cbdata);
int utofu_poll_mrq(utofu_vcq_hdl_t vcq_hdl, unsigned long flags, struct utofu_mrq_notice *notice);

#ifdef __cplusplus
}
#endif

#endif /* BINE_MPISHIM_UTOFU_H */
