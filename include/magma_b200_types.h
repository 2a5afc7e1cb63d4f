/*
 * magma_b200_types.h -- ABI types of the MAGMA C interface, kept identical so
 * that code compiled against MAGMA 2.2's headers links against libmagma_b200.
 *
 * Every definition here restates one in the reference's include/magma_types.h:
 *   magma_int_t (LP64 int)              include/magma_types.h:44-47
 *   opaque magma_queue_t                include/magma_types.h:73-74
 *   MAGMA_SUCCESS / MAGMA_ERR_* codes   include/magma_types.h:333-355
 *   trans / uplo / diag / side enums    include/magma_types.h:385-421
 * The numeric values are part of the ABI (callers pass them as ints), so they
 * must match exactly.
 */
#ifndef MAGMA_B200_TYPES_H
#define MAGMA_B200_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int magma_int_t;          /* LP64 build of MAGMA (include/magma_types.h:44-47) */
typedef int magma_index_t;
typedef magma_int_t magma_device_t;
typedef double real_Double_t;

/* Opaque queue (include/magma_types.h:73-74). The layout is private to the
 * library; callers only hold the pointer. */
struct magma_queue;
typedef struct magma_queue* magma_queue_t;

/* CUDA handle types, declared as the CUDA/cuBLAS headers declare them so this
 * header does not pull in the CUDA toolkit. */
#ifndef __DRIVER_TYPES_H__
typedef struct CUstream_st* cudaStream_t;
#endif
typedef struct cublasContext*   cublasHandle_t;
typedef struct cusparseContext* cusparseHandle_t;

typedef void*         magma_ptr;
typedef double*       magmaDouble_ptr;
typedef float*        magmaFloat_ptr;
typedef magma_int_t*  magmaInt_ptr;

/* Return codes (include/magma_types.h:333-355). */
#define MAGMA_SUCCESS               0
#define MAGMA_ERR                  -100
#define MAGMA_ERR_NOT_INITIALIZED  -101
#define MAGMA_ERR_NOT_SUPPORTED    -103
#define MAGMA_ERR_ILLEGAL_VALUE    -104
#define MAGMA_ERR_HOST_ALLOC       -112
#define MAGMA_ERR_DEVICE_ALLOC     -113
#define MAGMA_ERR_INVALID_PTR      -115
#define MAGMA_ERR_UNKNOWN          -116
#define MAGMA_ERR_NOT_IMPLEMENTED  -117
#define MAGMA_ERR_NAN              -118

typedef enum { MagmaFalse = 0, MagmaTrue = 1 } magma_bool_t;

typedef enum {
    MagmaNoTrans   = 111,
    MagmaTrans     = 112,
    MagmaConjTrans = 113
} magma_trans_t;

typedef enum {
    MagmaUpper = 121,
    MagmaLower = 122,
    MagmaFull  = 123
} magma_uplo_t;

typedef enum {
    MagmaNonUnit = 131,
    MagmaUnit    = 132
} magma_diag_t;

typedef enum {
    MagmaLeft  = 141,
    MagmaRight = 142
} magma_side_t;

#ifdef __cplusplus
}
#endif

#endif /* MAGMA_B200_TYPES_H */
