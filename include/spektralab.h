/* spektralab C ABI, B200 build.
 *
 * The drop-in boundary of the render path: the same entry points, status codes, limits and struct
 * layouts as the reference engine's public header (include/spektralab.h of the reference,
 * :19-392), so a host application or binding written against the reference links and runs against
 * this library unchanged. Each declaration names the reference line it mirrors.
 *
 * Conventions (reference include/spektralab.h:4-17):
 *   every entry point has C linkage; no exception crosses it
 *   failure: a negative spk_status or a NULL handle, with a message in the calling thread's
 *            last-error slot (spk_last_error)
 *   inputs are borrowed for the call; the engine copies what it keeps
 *   out_json strings are heap strings owned by the caller: spk_string_free(*out_json)
 *   calls on different sessions may run concurrently; calls on one session serialise on its lock
 *
 * B200 specifics:
 *   device          NULL or a pointer to an int holding a CUDA device ordinal (NULL: the current device)
 *   spk_image.data  host memory (pageable or pinned)
 *   spk_device_image.buffer  a CUDA device pointer on the engine's device
 *   spk_result      texture is an opaque handle owning the device RGBA16 image and a pinned host copy;
 *                   rgba16 points at the pinned host copy, rows of row_stride_px pixels (256-byte rows)
 */
#ifndef SPEKTRALAB_H
#define SPEKTRALAB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(SPK_BUILDING_LIBRARY)
#define SPK_API __attribute__((visibility("default")))
#else
#define SPK_API
#endif

/* versions (reference :30-36) */
#define SPK_TRANSPORT_VERSION 1
#define SPK_SCHEMA_VERSION 1
#define SPK_VERSION_MAJOR 1
#define SPK_VERSION_MINOR 0
#define SPK_VERSION_PATCH 0
#define SPK_VERSION_STRING "1.0.0"
#define SPK_ENGINE_NAME "spektralab.native"

/* status codes (reference :38-65) */
typedef int32_t spk_status;
#define SPK_OK 0
#define SPK_ERR_INVALID_ARG (-1) /* NULL required pointer, unknown tier */
#define SPK_ERR_USER (-2)        /* invalid parameter, stock, or a configuration that cannot be built */
#define SPK_ERR_RESOURCE (-3)    /* reserved */
#define SPK_ERR_UNSUPPORTED (-4) /* an entry point outside this build's render path */
#define SPK_ERR_GPU (-5)         /* device failure, out of memory, any render failure but a cancel */
#define SPK_ERR_IO (-6)          /* resource file missing or corrupt */
#define SPK_ERR_CANCELLED (-7)   /* the render was cancelled */
#define SPK_ERR_INTERNAL (-8)    /* a bug in the engine */

/* device types (reference :67-73) */
#define SPK_DEVICE_DESKTOP 0
#define SPK_DEVICE_PHONE 1
#define SPK_DEVICE_TABLET 2

/* limits (reference :75-76) */
#define SPK_MAX_PIXELS 151301008ULL /* 14204 x 10652 */

typedef struct spk_engine spk_engine;
typedef struct spk_session spk_session;

/* Host input image, row-major float32, channel c of pixel (x, y) at data[(y*width + x)*channels + c].
 * Size 24, alignment 8 (reference :83-95). */
typedef struct spk_image {
    const float* data;
    uint32_t width;
    uint32_t height;
    uint32_t channels; /* 3 or 4; a 4th channel is dropped */
} spk_image;

/* The same image in device memory: buffer is a CUDA device pointer (reference :97-106). */
typedef struct spk_device_image {
    void* buffer;
    uint32_t width;
    uint32_t height;
    uint32_t channels;
} spk_device_image;

/* One rendered image (reference :108-125). Channel c of pixel (x, y) is
 * rgba16[4 * (y * row_stride_px + x) + c]; alpha is 65535. Size 88, alignment 8. */
typedef struct spk_result {
    const uint16_t* rgba16;      /* pinned host pixels inside the texture handle */
    void* texture;               /* handle owning the device image and the host pixels, +1 */
    uint32_t width;
    uint32_t height;
    uint32_t row_stride_px;
    double elapsed_ms;
    int32_t reprint;
    int32_t negative_was_cached;
    char progress_id[40];
} spk_result;

#ifdef __cplusplus
#define SPK_STATIC_ASSERT(c, m) static_assert(c, m)
#define SPK_ALIGNOF(t) alignof(t)
#else
#define SPK_STATIC_ASSERT(c, m) _Static_assert(c, m)
#define SPK_ALIGNOF(t) _Alignof(t)
#endif

SPK_STATIC_ASSERT(sizeof(void*) == 8, "LP64 required");
SPK_STATIC_ASSERT(sizeof(spk_image) == 24 && SPK_ALIGNOF(spk_image) == 8, "spk_image layout");
SPK_STATIC_ASSERT(offsetof(spk_image, width) == 8 && offsetof(spk_image, channels) == 16, "spk_image fields");
SPK_STATIC_ASSERT(sizeof(spk_device_image) == 24 && SPK_ALIGNOF(spk_device_image) == 8, "spk_device_image layout");
SPK_STATIC_ASSERT(sizeof(spk_result) == 88 && SPK_ALIGNOF(spk_result) == 8, "spk_result layout");
SPK_STATIC_ASSERT(offsetof(spk_result, texture) == 8 && offsetof(spk_result, width) == 16, "spk_result fields");
SPK_STATIC_ASSERT(offsetof(spk_result, row_stride_px) == 24 && offsetof(spk_result, elapsed_ms) == 32, "spk_result fields");
SPK_STATIC_ASSERT(offsetof(spk_result, reprint) == 40 && offsetof(spk_result, negative_was_cached) == 44, "spk_result fields");
SPK_STATIC_ASSERT(offsetof(spk_result, progress_id) == 48, "spk_result.progress_id");

/* ---- engine lifecycle (reference :162-195) ---- */
SPK_API spk_engine* spk_engine_create(const char* resources_dir, void* device);             /* ref :181 */
SPK_API spk_engine* spk_engine_create_for_device(const char* resources_dir, void* device,
                                                 int32_t device_type);                       /* ref :182 */
SPK_API void spk_engine_destroy(spk_engine* engine);                                         /* ref :189 */
SPK_API size_t spk_engine_trim(spk_engine* engine);                                          /* ref :194 */
SPK_API const char* spk_build_info(void);                                                    /* ref :198 */

/* ---- introspection (reference :200-215) ---- */
SPK_API const char* spk_capabilities(spk_engine* engine);                                    /* ref :205 */
SPK_API const char* spk_params_schema(spk_engine* engine);                                   /* ref :209 */
SPK_API const char* spk_memory_report(spk_engine* engine);                                   /* ref :213 */
SPK_API spk_status spk_warm_up(spk_engine* engine, const char* film_stock, const char* print_stock,
                               char** out_json);                                             /* ref :228 */

/* ---- sessions (reference :231-286) ---- */
SPK_API spk_session* spk_open(spk_engine* engine, const spk_image* input, const char* params_delta_json,
                              char** out_json);                                              /* ref :248 */
SPK_API spk_session* spk_open_device(spk_engine* engine, const spk_device_image* input,
                                     const char* params_delta_json, char** out_json);        /* ref :254 */
SPK_API spk_status spk_set_params(spk_session* session, const char* params_delta_json,
                                  char** out_json);                                          /* ref :269 */
SPK_API spk_status spk_get_params(spk_session* session, char** out_json);                    /* ref :276 */
SPK_API void spk_session_release(spk_session* session);                                      /* ref :282 */

/* ---- rendering (reference :284-308) ---- */
SPK_API spk_status spk_render(spk_session* session, const char* tier, spk_result* out);      /* ref :294 */
SPK_API spk_status spk_reprint(spk_session* session, const char* tier, spk_result* out);     /* ref :302 */
SPK_API void spk_result_free(spk_result* result);                                            /* ref :308 */

/* ---- outside the render path: present for link compatibility (reference :310-361) ---- */
SPK_API spk_status spk_solve(spk_session* session, const char* target, char** out_json);     /* ref :321 */
SPK_API const char* spk_print_lut_catalog(spk_engine* engine);                               /* ref :327 */
SPK_API spk_status spk_print_lut_table(spk_engine* engine, const char* print_stock, const float** out_table,
                                       uint32_t* out_size);                                  /* ref :333 */
SPK_API spk_status spk_preview_stock_lut(spk_session* session, const char* print_stock, const char* tier,
                                         spk_result* out, char** out_json);                  /* ref :345 */
SPK_API spk_status spk_output_transform(spk_engine* engine, const char* src_cs, const char* dst_cs,
                                        const char* gamut_compress_json, char** out_json,
                                        const float** out_cmax, uint32_t* out_cmax_count);   /* ref :359 */

/* ---- control (reference :363-386) ---- */
SPK_API void spk_cancel(spk_session* session, const char* progress_id);                      /* ref :369 */
SPK_API spk_status spk_progress(spk_session* session, const char* progress_id, char** out_json); /* ref :375 */
SPK_API void spk_string_free(char* s);                                                       /* ref :379 */
SPK_API const char* spk_last_error(spk_engine* engine);                                      /* ref :385 */

#ifdef __cplusplus
}
#endif

#endif /* SPEKTRALAB_H */
