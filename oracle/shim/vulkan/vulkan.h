/* Oracle build shim (test infrastructure only).
 *
 * The reference's host-memory descriptor (include/core/drivers/memory.hpp:7 ->
 * include/core/drivers/vulkan/buffer.hpp) names three Vulkan handle types. The CPU
 * path never touches them, so this header declares the names and nothing else.
 * No Vulkan library is loaded or needed. */
#pragma once
#include <stdint.h>
typedef struct VkBuffer_T *VkBuffer;
typedef struct VkDeviceMemory_T *VkDeviceMemory;
#define VK_NULL_HANDLE nullptr
