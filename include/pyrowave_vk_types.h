/*
 * Minimal stand-ins for the Vulkan types that appear in pyrowave.h.
 *
 * The reference's pyrowave.h refuses to compile unless the Vulkan headers were
 * included first (its Vulkan-facing entry points take VkImage, VkSemaphore,
 * ...). This implementation has no Vulkan path, so when the real headers are
 * absent these opaque declarations stand in for them: handles are pointers to
 * incomplete structs (the Vulkan ABI for both dispatchable and, on 64-bit
 * targets, non-dispatchable handles), enums are 32-bit integers, and the
 * create-info structs are only ever passed by pointer. The struct layouts of
 * pyrowave.h therefore match a build against the real headers.
 *
 * If the application includes <vulkan/vulkan.h> before pyrowave.h, this file
 * is not used.
 */
#ifndef PYROWAVE_VK_TYPES_H_
#define PYROWAVE_VK_TYPES_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct VkInstance_T *VkInstance;
typedef struct VkPhysicalDevice_T *VkPhysicalDevice;
typedef struct VkDevice_T *VkDevice;
typedef struct VkQueue_T *VkQueue;
typedef struct VkCommandBuffer_T *VkCommandBuffer;
typedef struct VkImage_T *VkImage;
typedef struct VkSemaphore_T *VkSemaphore;

typedef uint32_t VkFlags;
typedef VkFlags VkSemaphoreImportFlags;
typedef int32_t VkFormat;
typedef int32_t VkImageLayout;
typedef int32_t VkImageAspectFlagBits;
typedef int32_t VkComponentSwizzle;
typedef int32_t VkQueueFlagBits;
typedef int32_t VkImageUsageFlagBits;
typedef int32_t VkSemaphoreType;
typedef int32_t VkExternalSemaphoreHandleTypeFlagBits;
typedef int32_t VkExternalMemoryHandleTypeFlagBits;

typedef struct VkInstanceCreateInfo VkInstanceCreateInfo;
typedef struct VkDeviceCreateInfo VkDeviceCreateInfo;
typedef struct VkImageCreateInfo VkImageCreateInfo;

typedef void (*PFN_vkVoidFunction)(void);
typedef PFN_vkVoidFunction (*PFN_vkGetInstanceProcAddr)(VkInstance instance, const char *pName);

#ifndef VK_UUID_SIZE
#define VK_UUID_SIZE 16U
#endif
#ifndef VK_LUID_SIZE
#define VK_LUID_SIZE 8U
#endif
#ifndef VK_NULL_HANDLE
#define VK_NULL_HANDLE 0
#endif

#ifdef __cplusplus
}
#endif

#endif
