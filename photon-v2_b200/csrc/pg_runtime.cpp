#include "pg_runtime.h"

#include <mutex>

namespace pg
{

namespace
{
thread_local std::string t_last_error;
}

void set_last_error(const std::string& message)
{
	t_last_error = message;
}

const char* last_error()
{
	return t_last_error.c_str();
}

void require_device()
{
	int n = 0;
	const cudaError_t err = cudaGetDeviceCount(&n);
	if(err != cudaSuccess || n == 0)
	{
		throw Error(PG_ERR_NO_DEVICE,
			std::string("no CUDA device available (") + cudaGetErrorString(err) +
			"); the B200 path-tracing core has no CPU fallback");
	}
}

int current_device()
{
	int dev = -1;
	PG_CUDA_CHECK(cudaGetDevice(&dev));
	if(dev < 0 || dev >= kMaxDevices)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "device index " + std::to_string(dev) + " out of range");
	}
	return dev;
}

cudaStream_t library_stream()
{
	static std::mutex mutex;
	static cudaStream_t streams[kMaxDevices] = {};
	const int dev = current_device();
	std::lock_guard<std::mutex> lock(mutex);
	if(!streams[dev])
	{
		const cudaError_t status = cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
		if(status != cudaSuccess)
		{
			streams[dev] = nullptr;
			cudaGetLastError();
			throw Error(PG_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(status));
		}
	}
	return streams[dev];
}

void check_same_device(int owner_device, int current, const char* what)
{
	if(current != owner_device)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, std::string(what) + " lives on device " + std::to_string(owner_device) +
		            " but device " + std::to_string(current) + " is current; make its device current first");
	}
}

void require_same_device(int owner_device, const char* what)
{
	check_same_device(owner_device, current_device(), what);
}

int sm_count()
{
	int dev = 0;
	PG_CUDA_CHECK(cudaGetDevice(&dev));
	int n = 0;
	PG_CUDA_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
	return n;
}

}// end namespace pg
