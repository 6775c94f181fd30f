/* Primitive types and small structs of the Photon C API, as the B200 library exports it.
 *
 * Same names, sizes and enumerator values as the reference's
 * Engine/CEngine/Include/ph_c_core_types.h:8-86, so that a program compiled against the reference
 * header links against libphoton_gpu.so unchanged. */
#ifndef PH_C_CORE_TYPES_H
#define PH_C_CORE_TYPES_H

#include <stddef.h>
#include <stdint.h>

typedef int8_t         PhInt8;
typedef uint8_t        PhUInt8;
typedef int16_t        PhInt16;
typedef uint16_t       PhUInt16;
typedef int32_t        PhInt32;
typedef uint32_t       PhUInt32;
typedef int64_t        PhInt64;
typedef uint64_t       PhUInt64;
typedef float          PhFloat32;
typedef double         PhFloat64;
typedef char           PhChar;
typedef unsigned char  PhUChar;
typedef size_t         PhSize;

typedef enum PhBool { PH_FALSE, PH_TRUE } PhBool;

typedef enum PhEndian { PH_NATIVE_ENDIAN, PH_LITTLE_ENDIAN, PH_BIG_ENDIAN } PhEndian;

typedef enum PhBufferFormat
{
	PH_BUFFER_FORMAT_EXR_IMAGE,
	PH_BUFFER_FORMAT_FLOAT32_ARRAY
} PhBufferFormat;

typedef enum PhFrameRegionStatus
{
	PH_FRAME_REGION_STATUS_INVALID,
	PH_FRAME_REGION_STATUS_FINISHED,
	PH_FRAME_REGION_STATUS_UPDATING
} PhFrameRegionStatus;

typedef struct PhRenderProgress
{
	PhUInt64 totalWork;
	PhUInt64 workDone;
	PhUInt64 elapsedMs;
} PhRenderProgress;

typedef struct PhFrameRegionInfo
{
	PhUInt32 xPx;
	PhUInt32 yPx;
	PhUInt32 widthPx;
	PhUInt32 heightPx;
	PhFrameRegionStatus status;
} PhFrameRegionInfo;

#define PH_MAX_FRAME_DATA_NAME_SIZE 256

typedef struct PhFrameSaveInfo
{
	PhSize numChannels;
	const PhChar* const* channelNames;
	PhEndian endianness;
} PhFrameSaveInfo;

#endif /* PH_C_CORE_TYPES_H */
