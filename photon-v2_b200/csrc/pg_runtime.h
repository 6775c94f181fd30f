// Runtime plumbing shared by the C ABI entry points: per-thread error messages, CUDA error
// checks, the id -> object registries and the library stream.
#pragma once

#include "pg_common.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>

namespace pg
{

// Exception carrying a status code; caught at the C ABI boundary.
struct Error : std::runtime_error
{
	int status;
	Error(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

void set_last_error(const std::string& message);
const char* last_error();

#define PG_CUDA_CHECK(expr)                                                                          \
	do                                                                                               \
	{                                                                                                \
		const cudaError_t pg_err_ = (expr);                                                          \
		if(pg_err_ != cudaSuccess)                                                                   \
		{                                                                                            \
			throw ::pg::Error(::pg::PG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(pg_err_)); \
		}                                                                                            \
	} while(0)

// Runs `fn` and converts exceptions into a status code + thread-local message.
template<typename Fn>
int guarded(Fn&& fn)
{
	try
	{
		fn();
		set_last_error("");
		return PG_OK;
	}
	catch(const Error& e)
	{
		set_last_error(e.what());
		return e.status;
	}
	catch(const std::exception& e)
	{
		set_last_error(e.what());
		return PG_ERR_INVALID_ARGUMENT;
	}
	catch(...)
	{
		set_last_error("unknown error");
		return PG_ERR_INVALID_ARGUMENT;
	}
}

// Fails loudly when no CUDA device is usable: the library has no CPU fallback.
void require_device();

// Devices the library keeps per-device state for (streams, launch shapes, static scratch).
constexpr int kMaxDevices = 64;

// The current CUDA device (checked against kMaxDevices).
int current_device();

// The stream library work of the current device is issued on (one per device, created on first
// use with that device current).
cudaStream_t library_stream();

// Throws PG_ERR_INVALID_ARGUMENT unless `owner_device` is the current device: objects (geometry,
// scenes) stay on the device that was current when they were created, and every call on them
// must be made with that device current.
void require_same_device(int owner_device, const char* what);
// The comparison itself, for a given current device.
void check_same_device(int owner_device, int current, const char* what);

// Thread-safe id -> object table, ids start at 1 (0 is never valid).
template<typename T>
class Registry
{
public:
	uint64_t add(std::unique_ptr<T> obj)
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		const uint64_t id = ++m_next;
		m_items[id] = std::shared_ptr<T>(std::move(obj));
		return id;
	}

	std::shared_ptr<T> get(uint64_t id)
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		auto it = m_items.find(id);
		return it == m_items.end() ? nullptr : it->second;
	}

	bool remove(uint64_t id)
	{
		std::shared_ptr<T> victim;
		{
			std::lock_guard<std::mutex> lock(m_mutex);
			auto it = m_items.find(id);
			if(it == m_items.end())
			{
				return false;
			}
			victim = std::move(it->second);
			m_items.erase(it);
		}
		return true;
	}

private:
	std::mutex m_mutex;
	uint64_t m_next = 0;
	std::unordered_map<uint64_t, std::shared_ptr<T>> m_items;
};

// A CUDA event destroyed with its scope, so that a CUDA check that throws between the event's
// creation and its last use does not leak it.
class ScopedEvent
{
public:
	ScopedEvent() { PG_CUDA_CHECK(cudaEventCreate(&m_event)); }
	~ScopedEvent() { cudaEventDestroy(m_event); }
	ScopedEvent(const ScopedEvent&) = delete;
	ScopedEvent& operator=(const ScopedEvent&) = delete;
	cudaEvent_t get() const { return m_event; }

private:
	cudaEvent_t m_event = nullptr;
};

// Device buffer with RAII ownership.
template<typename T>
class DeviceBuffer
{
public:
	DeviceBuffer() = default;
	explicit DeviceBuffer(std::size_t n) { resize(n); }
	~DeviceBuffer() { release(); }
	DeviceBuffer(const DeviceBuffer&) = delete;
	DeviceBuffer& operator = (const DeviceBuffer&) = delete;
	DeviceBuffer(DeviceBuffer&& o) noexcept : m_ptr(o.m_ptr), m_size(o.m_size) { o.m_ptr = nullptr; o.m_size = 0; }
	DeviceBuffer& operator = (DeviceBuffer&& o) noexcept
	{
		if(this != &o)
		{
			release();
			m_ptr = o.m_ptr; m_size = o.m_size;
			o.m_ptr = nullptr; o.m_size = 0;
		}
		return *this;
	}

	void resize(std::size_t n)
	{
		if(n == m_size)
		{
			return;
		}
		release();
		if(n > 0)
		{
			PG_CUDA_CHECK(cudaMalloc(reinterpret_cast<void**>(&m_ptr), n * sizeof(T)));
		}
		m_size = n;
	}

	void release()
	{
		if(m_ptr)
		{
			cudaFree(m_ptr);
			m_ptr = nullptr;
		}
		m_size = 0;
	}

	T* get() const { return m_ptr; }
	std::size_t size() const { return m_size; }
	std::size_t bytes() const { return m_size * sizeof(T); }

private:
	T* m_ptr = nullptr;
	std::size_t m_size = 0;
};

// Number of SMs of the current device (grid sizing).
int sm_count();

}// end namespace pg
