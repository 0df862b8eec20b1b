/*
 * PyroWave C API, B200 (CUDA) implementation.
 *
 * Every declaration keeps the name, argument meaning, struct layout and result
 * codes of the reference's public header (pyrowave.h of Themaister/pyrowave,
 * API 0.4.0), so existing callers relink against libpyrowave-shared.so.0
 * unchanged. Each entry point cites the reference declaration it replaces.
 *
 * Behaviour on this implementation:
 *   - Encode/decode run as sm_100a CUDA kernels on the current CUDA device.
 *   - The CPU-buffer entry points are complete drop-ins.
 *   - Entry points whose only purpose is Vulkan interop (external semaphores,
 *     external images, borrowed command buffers, Vulkan device import) return
 *     PYROWAVE_ERROR_NOT_IMPLEMENTED / NULL handles; the equivalent CUDA-stream
 *     and device-pointer path is declared in pyrowave_cuda.h.
 */
#ifndef PYROWAVE_H_
#define PYROWAVE_H_

#if !defined(VULKAN_CORE_H_)
#include "pyrowave_vk_types.h"
#endif

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#else
#include <stdbool.h>
#endif

#define PYROWAVE_API_VERSION_MAJOR 0
#define PYROWAVE_API_VERSION_MINOR 4
#define PYROWAVE_API_VERSION_PATCH 0

#if defined(PYROWAVE_EXPORT_SYMBOLS) && defined(__GNUC__)
#define PYROWAVE_PUBLIC_API __attribute__((visibility("default")))
#else
#define PYROWAVE_PUBLIC_API
#endif

typedef void (*pyrowave_message_cb)(void *userdata, const char *msg);

/* Result codes: reference pyrowave.h:43-56. */
typedef enum pyrowave_result
{
	PYROWAVE_SUCCESS = 0,
	PYROWAVE_TIMEOUT = 1,
	PYROWAVE_ERROR_GENERIC = -1,
	PYROWAVE_ERROR_INVALID_ARGUMENT = -2,
	PYROWAVE_ERROR_OUT_OF_HOST_MEMORY = -3,
	PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY = -4,
	PYROWAVE_ERROR_NO_VULKAN = -5,
	PYROWAVE_ERROR_NOT_IMPLEMENTED = -6,
	PYROWAVE_ERROR_UNSUPPORTED_EXTERNAL_HANDLE = -7,
	PYROWAVE_ERROR_FAILED_EXTERNAL_HANDLE = -8,
	PYROWAVE_ERROR_INT_MAX = 0x7fffffff
} pyrowave_result;

/* reference pyrowave.h:58-63 */
typedef enum pyrowave_chroma_subsampling
{
	PYROWAVE_CHROMA_SUBSAMPLING_420 = 0,
	PYROWAVE_CHROMA_SUBSAMPLING_444 = 1,
	PYROWAVE_CHROMA_SUBSAMPLING_INT_MAX = 0x7fffffff
} pyrowave_chroma_subsampling;

typedef struct pyrowave_encoder_opaque *pyrowave_encoder;
typedef struct pyrowave_decoder_opaque *pyrowave_decoder;
typedef struct pyrowave_device_opaque *pyrowave_device;
typedef struct pyrowave_sync_object_opaque *pyrowave_sync_object;
typedef struct pyrowave_image_opaque *pyrowave_image;

/* reference pyrowave.h:73 */
PYROWAVE_PUBLIC_API void pyrowave_get_api_version(uint32_t *major, uint32_t *minor, uint32_t *patch);

/* reference pyrowave.h:76. Binds the current CUDA device. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_create_default_device(pyrowave_device *device);

/* reference pyrowave.h:78-83 */
typedef struct pyrowave_device_create_queue_info
{
	VkQueue queue;
	uint32_t familyIndex;
	uint32_t index;
} pyrowave_device_create_queue_info;

typedef void (*pyrowave_queue_lock_cb)(void *userdata);

/* reference pyrowave.h:89-125 */
typedef struct pyrowave_device_create_info
{
	PFN_vkGetInstanceProcAddr GetInstanceProcAddr;
	VkInstance instance;
	VkPhysicalDevice physical_device;
	VkDevice device;
	const VkInstanceCreateInfo *instance_create_info;
	const VkDeviceCreateInfo *device_create_info;
	pyrowave_device_create_queue_info *queue_info;
	uint32_t queue_info_count;
	pyrowave_queue_lock_cb queue_lock_callback;
	pyrowave_queue_lock_cb queue_unlock_callback;
	void *userdata;
} pyrowave_device_create_info;

typedef struct pyrowave_uuid
{
	uint8_t uuid[VK_UUID_SIZE];
} pyrowave_uuid;

typedef struct pyrowave_luid
{
	uint8_t luid[VK_LUID_SIZE];
} pyrowave_luid;

/* reference pyrowave.h:152-153. Importing a VkDevice: PYROWAVE_ERROR_NO_VULKAN. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_create_device(const pyrowave_device_create_info *info, pyrowave_device *device);

/* reference pyrowave.h:156-163. Matches on the CUDA device's PCI vendor/device
 * id and UUID where given; otherwise the current CUDA device. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_create_device_by_compat(uint32_t vid, uint32_t pid,
                                                                     const pyrowave_uuid *device_uuid,
                                                                     const pyrowave_uuid *driver_uuid,
                                                                     const pyrowave_luid *device_luid,
                                                                     pyrowave_device *device);

/* reference pyrowave.h:166-167. Per-stage GPU time ("DWT", "Quant", ...) from CUDA events. */
PYROWAVE_PUBLIC_API void pyrowave_device_report_performance_stats(pyrowave_device device, pyrowave_message_cb cb,
                                                                  void *userdata, bool reset);

/* reference pyrowave.h:170-173. Writes VK_NULL_HANDLE. */
PYROWAVE_PUBLIC_API void pyrowave_device_get_vk_device_handles(pyrowave_device device, VkInstance *vk_instance,
                                                               VkPhysicalDevice *vk_physical_device, VkDevice *vk_device);

/* reference pyrowave.h:184-185. No-op (there are no Vulkan command buffers). */
PYROWAVE_PUBLIC_API void pyrowave_device_set_command_buffer(pyrowave_device device, VkCommandBuffer cmd);

/* reference pyrowave.h:197-198. Accepted and ignored: work goes to the device's CUDA stream. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_device_set_queue_type(pyrowave_device device, VkQueueFlagBits queue_flags);

/* reference pyrowave.h:200-201. Returns false. */
PYROWAVE_PUBLIC_API bool pyrowave_device_confirm_interop_support(pyrowave_device device);

/* reference pyrowave.h:204 */
PYROWAVE_PUBLIC_API void pyrowave_device_destroy(pyrowave_device device);

typedef uintptr_t pyrowave_os_handle;

/* reference pyrowave.h:212-243 */
typedef struct pyrowave_sync_object_create_info
{
	pyrowave_device device;
	pyrowave_os_handle external_handle;
	VkExternalSemaphoreHandleTypeFlagBits handle_type;
	VkSemaphoreType semaphore_type;
	VkSemaphoreImportFlags import_flags;
} pyrowave_sync_object_create_info;

/* reference pyrowave.h:245-266: external semaphores, PYROWAVE_ERROR_NOT_IMPLEMENTED. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_sync_object_create(const pyrowave_sync_object_create_info *info,
                                                                pyrowave_sync_object *sync);
PYROWAVE_PUBLIC_API VkSemaphore pyrowave_sync_object_get_semaphore(pyrowave_sync_object sync);
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_sync_object_export_handle(pyrowave_sync_object sync,
                                                                       pyrowave_os_handle *handle);
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_sync_object_cpu_wait(pyrowave_sync_object sync, uint64_t value,
                                                                  uint64_t timeout);
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_sync_object_cpu_signal(pyrowave_sync_object sync, uint64_t value);
PYROWAVE_PUBLIC_API void pyrowave_sync_object_destroy(pyrowave_sync_object sync);

/* reference pyrowave.h:270-295 */
typedef struct pyrowave_image_view
{
	VkImage image;
	uint32_t width;
	uint32_t height;
	VkFormat image_format;
	VkFormat view_format;
	uint32_t mip_level;
	uint32_t layer;
	VkImageAspectFlagBits aspect;
	VkComponentSwizzle swizzle;
	VkImageLayout layout;
} pyrowave_image_view;

/* reference pyrowave.h:297-326 */
typedef struct pyrowave_image_create_info
{
	pyrowave_device device;
	pyrowave_os_handle external_handle;
	VkExternalMemoryHandleTypeFlagBits handle_type;
	const VkImageCreateInfo *image_create_info;
} pyrowave_image_create_info;

/* reference pyrowave.h:330-351: external images, PYROWAVE_ERROR_NOT_IMPLEMENTED. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_image_create(const pyrowave_image_create_info *info, pyrowave_image *image);
PYROWAVE_PUBLIC_API VkImage pyrowave_image_get_handle(pyrowave_image image);
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_image_get_image_view(pyrowave_image image, VkImageAspectFlagBits aspect,
                                                                  VkImageUsageFlagBits usage, pyrowave_image_view *view);
PYROWAVE_PUBLIC_API void pyrowave_image_destroy(pyrowave_image image);

/* reference pyrowave.h:355-362 */
typedef struct pyrowave_encoder_create_info
{
	pyrowave_device device;
	int width;  /* even for 4:2:0 */
	int height; /* even for 4:2:0 */
	pyrowave_chroma_subsampling chroma;
} pyrowave_encoder_create_info;

/* reference pyrowave.h:364-368 */
typedef struct pyrowave_packet
{
	size_t offset;
	size_t size;
} pyrowave_packet;

/* reference pyrowave.h:370-407 */
typedef struct pyrowave_sync_point
{
	VkSemaphore semaphore;
	uint64_t value;
} pyrowave_sync_point;

typedef struct pyrowave_gpu_external_reference
{
	pyrowave_image image;
	uint32_t queue_family_index;
} pyrowave_gpu_external_reference;

typedef struct pyrowave_gpu_buffers
{
	pyrowave_image_view planes[3];
} pyrowave_gpu_buffers;

typedef struct pyrowave_gpu_sync_operation
{
	const pyrowave_gpu_external_reference *images;
	size_t num_images;
	pyrowave_sync_point sync;
} pyrowave_gpu_sync_operation;

/* reference pyrowave.h:412-418 */
typedef enum pyrowave_cpu_buffer_format
{
	PYROWAVE_CPU_BUFFER_FORMAT_NV12 = 0,    /* Y, then interleaved CbCr (encode only) */
	PYROWAVE_CPU_BUFFER_FORMAT_YUV420P = 1,
	PYROWAVE_CPU_BUFFER_FORMAT_YUV444P = 2,
	PYROWAVE_CPU_BUFFER_FORMAT_INT_MAX = 0x7fffffff
} pyrowave_cpu_buffer_format;

/* reference pyrowave.h:420-433 */
typedef struct pyrowave_cpu_buffer
{
	void *data[3];
	size_t row_stride_in_bytes[3];
	size_t plane_size_in_bytes[3];
	int width;
	int height;
	pyrowave_cpu_buffer_format format;
} pyrowave_cpu_buffer;

/* reference pyrowave.h:435-439 */
typedef struct pyrowave_rate_control
{
	size_t maximum_bitstream_size;
} pyrowave_rate_control;

/* reference pyrowave.h:442-443. Not thread safe per encoder. Errors:
 * INVALID_ARGUMENT (no device, non-positive or odd 4:2:0 size), GENERIC (init). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_encoder_create(const pyrowave_encoder_create_info *info,
                                                            pyrowave_encoder *encoder);

/* reference pyrowave.h:457-462. Vulkan images: PYROWAVE_ERROR_NOT_IMPLEMENTED
 * (use pyrowave_cuda_encoder_encode). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_encoder_encode_gpu_synchronous(pyrowave_encoder encoder,
                                                                            const pyrowave_gpu_sync_operation *acquire,
                                                                            const pyrowave_gpu_sync_operation *release,
                                                                            const pyrowave_gpu_buffers *buffers,
                                                                            const pyrowave_rate_control *rate_control);

/* reference pyrowave.h:465-467. Queues the encode and returns; the following
 * compute_num_packets / packetize wait for it. Clobbers the previous frame. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_encoder_encode_cpu_synchronous(pyrowave_encoder encoder,
                                                                            const pyrowave_cpu_buffer *buffers,
                                                                            const pyrowave_rate_control *rate_control);

/* reference pyrowave.h:471-472. GENERIC if nothing was encoded yet. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_encoder_compute_num_packets(pyrowave_encoder encoder,
                                                                         size_t packet_boundary, size_t *num_packets);

/* reference pyrowave.h:475-477 */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_encoder_packetize(pyrowave_encoder encoder, pyrowave_packet *packets,
                                                               size_t packet_boundary, size_t *out_packets,
                                                               void *bitstream, size_t size);

/* reference pyrowave.h:480-481 */
PYROWAVE_PUBLIC_API void pyrowave_encoder_destroy(pyrowave_encoder encoder);

/* reference pyrowave.h:485-493 */
typedef struct pyrowave_decoder_create_info
{
	pyrowave_device device;
	int width;
	int height;
	pyrowave_chroma_subsampling chroma;
	bool fragment_path;
} pyrowave_decoder_create_info;

/* reference pyrowave.h:498-499. Always false (compute path only). */
PYROWAVE_PUBLIC_API bool pyrowave_decoder_device_prefers_fragment_path(pyrowave_device device);

/* reference pyrowave.h:501-502. fragment_path is accepted and ignored. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_decoder_create(const pyrowave_decoder_create_info *info,
                                                            pyrowave_decoder *decoder);

/* reference pyrowave.h:505 */
PYROWAVE_PUBLIC_API void pyrowave_decoder_clear(pyrowave_decoder decoder);

/* reference pyrowave.h:511-512. INVALID_ARGUMENT on a malformed packet. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_decoder_push_packet(pyrowave_decoder decoder, const void *data,
                                                                 size_t size);

/* reference pyrowave.h:515-516 */
PYROWAVE_PUBLIC_API bool pyrowave_decoder_decode_is_ready(pyrowave_decoder decoder, bool allow_partial_frame);

/* reference pyrowave.h:528-532. Vulkan images: PYROWAVE_ERROR_NOT_IMPLEMENTED
 * (use pyrowave_cuda_decoder_decode). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_decoder_decode_gpu_buffer(pyrowave_decoder decoder,
                                                                       const pyrowave_gpu_sync_operation *acquire,
                                                                       const pyrowave_gpu_sync_operation *release,
                                                                       const pyrowave_gpu_buffers *buffers);

/* reference pyrowave.h:535-536. Fully synchronous. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_decoder_decode_cpu_buffer_synchronous(pyrowave_decoder decoder,
                                                                                   const pyrowave_cpu_buffer *buffers);

/* reference pyrowave.h:539 */
PYROWAVE_PUBLIC_API void pyrowave_decoder_destroy(pyrowave_decoder decoder);

#ifdef __cplusplus
}
#endif

#endif
