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

cudaStream_t library_stream()
{
	static std::once_flag once;
	static cudaStream_t stream = nullptr;
	static cudaError_t status = cudaSuccess;
	std::call_once(once, []
	{
		status = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
	});
	if(status != cudaSuccess)
	{
		throw Error(PG_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(status));
	}
	return stream;
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
