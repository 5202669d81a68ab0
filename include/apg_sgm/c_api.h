/* apg-sgm session C API, served by the B200 engine (libapg_sgm_b200.so).
 *
 * Drop-in for the reference's include/apg_sgm/c_api.h (lines 27-102 there): the same symbols,
 * constants, struct layouts and status codes, so a C caller links against this library instead
 * of the CPU one without source changes.  Semantics are the reference's (src/c_api.cpp:10-204):
 * borrowed strided inputs, result-owned outputs valid until the next process/destroy, per-session
 * last_error, frame counter and accumulated wall time, struct_size ABI check, no exception ever
 * crosses the ABI.
 *
 * Backend field: the reference knows 0 = Auto, 1 = Dense, 2 = Packed and maps any other value to
 * Auto.  Here every value runs the CUDA engine (value 3, APG_BACKEND_CUDA, names it explicitly);
 * Dense and Packed are bit-identical in the reference, so there is nothing to choose between.
 */
#ifndef APG_SGM_C_API_H
#define APG_SGM_C_API_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__) && __GNUC__ >= 4
#define APG_API __attribute__((visibility("default")))
#else
#define APG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define APG_QUALITY_FAST 0
#define APG_QUALITY_BALANCED 1
#define APG_QUALITY_HIGH_QUALITY 2

#define APG_MEMORY_RELEASE_PER_FRAME 0
#define APG_MEMORY_BOUNDED_REUSE 1

#define APG_BACKEND_AUTO 0
#define APG_BACKEND_DENSE 1
#define APG_BACKEND_PACKED 2
#define APG_BACKEND_CUDA 3 /* new: explicit CUDA engine (every value runs it in this library) */

typedef enum {
    APG_STATUS_OK = 0,
    APG_STATUS_EMPTY_INPUT = 1,
    APG_STATUS_SIZE_MISMATCH = 2,
    APG_STATUS_INVALID_DISPARITY_RANGE = 3,
    APG_STATUS_INVALID_CONFIG = 4,
    APG_STATUS_UNSUPPORTED_BACKEND = 5,
    APG_STATUS_RESOURCE_LIMIT_EXCEEDED = 6,
    APG_STATUS_ALLOCATION_FAILURE = 7,
    APG_STATUS_INTERNAL_ERROR = 8
} apg_status_code_t;

typedef struct {
    const uint8_t* data;
    int width;
    int height;
    int stride;   /* bytes between rows, >= width * channels */
    int channels; /* 1 (gray) or 3 (RGB) */
} apg_image_view_t;

typedef struct apg_session_s* apg_session_t;
typedef struct apg_result_s* apg_result_t;

typedef struct {
    uint32_t struct_size;      /* 0 or sizeof(apg_session_options_t) */
    int quality_mode;          /* APG_QUALITY_* */
    int memory_policy;         /* APG_MEMORY_* */
    size_t max_retained_bytes; /* 0 = unconstrained */
    int num_threads;           /* accepted for compatibility; the CUDA engine ignores it */
    int backend;               /* APG_BACKEND_* */
    int min_disparity;
    int max_disparity;         /* <= min_disparity selects 128 */
} apg_session_options_t;

APG_API apg_session_t apg_session_create(int quality_mode, int memory_policy);
APG_API apg_session_t apg_session_create_ex(const apg_session_options_t* options);
APG_API void apg_session_destroy(apg_session_t session);
APG_API void apg_session_reset(apg_session_t session);

APG_API apg_result_t apg_result_create(void);
APG_API void apg_result_destroy(apg_result_t result);

APG_API int apg_session_process(apg_session_t session, const apg_image_view_t* left, const apg_image_view_t* right,
                                apg_result_t result);

APG_API const float* apg_result_get_disparity(apg_result_t result, int* width, int* height);
APG_API const float* apg_result_get_confidence(apg_result_t result, int* width, int* height);
APG_API const uint8_t* apg_result_get_invalid_reason(apg_result_t result, int* width, int* height);
APG_API const uint8_t* apg_result_get_reliable_mask(apg_result_t result, int* width, int* height);

APG_API const char* apg_session_get_last_error(apg_session_t session);
APG_API size_t apg_session_get_allocated_bytes(apg_session_t session);
APG_API size_t apg_session_get_frame_count(apg_session_t session);
APG_API double apg_session_get_total_time_ms(apg_session_t session);

APG_API const char* apg_status_string(int status_code);
APG_API const char* apg_version_string(void);

#ifdef __cplusplus
}
#endif

#endif /* APG_SGM_C_API_H */
