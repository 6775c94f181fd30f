// Oracle build shim (test infrastructure only, never linked into the product).
//
// The reference engine includes <moodycamel/concurrentqueue.h>, a third-party header that is
// not vendored with the reference sources. Only a tiny subset of its interface is used by
// Engine/Source/Utility/Concurrent/TAtomicQuasiQueue.ipp:13-67 (enqueue, enqueue_bulk,
// try_enqueue, try_dequeue, try_dequeue_bulk, size_approx, is_lock_free). This header provides
// that subset as a mutex-guarded deque. It is semantically a FIFO, which satisfies the
// "mostly FIFO" contract stated in TAtomicQuasiQueue.h; throughput is irrelevant because the
// queue only carries work descriptors, never per-sample data.
#pragma once

#include <cstddef>
#include <deque>
#include <mutex>
#include <utility>

namespace moodycamel
{

template<typename T>
class ConcurrentQueue
{
public:
	ConcurrentQueue() = default;
	explicit ConcurrentQueue(std::size_t /*initialCapacity*/) {}

	// The reference move-assigns whole queues when it resets renderer state; the mutex itself
	// is not moved, only the queued items.
	ConcurrentQueue(ConcurrentQueue&& other)
	{
		std::lock_guard<std::mutex> lock(other.m_mutex);
		m_items = std::move(other.m_items);
	}

	ConcurrentQueue& operator = (ConcurrentQueue&& other)
	{
		if(this != &other)
		{
			std::scoped_lock lock(m_mutex, other.m_mutex);
			m_items = std::move(other.m_items);
		}
		return *this;
	}

	// The reference static_asserts lock-freedom; the shim reports true so the header compiles.
	static constexpr bool is_lock_free() { return true; }

	template<typename U>
	bool enqueue(U&& item)
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		m_items.emplace_back(std::forward<U>(item));
		return true;
	}

	template<typename It>
	bool enqueue_bulk(It first, std::size_t count)
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		for(std::size_t i = 0; i < count; ++i, ++first)
		{
			m_items.emplace_back(*first);
		}
		return true;
	}

	template<typename U>
	bool try_enqueue(U&& item)
	{
		return enqueue(std::forward<U>(item));
	}

	template<typename U>
	bool try_dequeue(U& out)
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		if(m_items.empty())
		{
			return false;
		}
		out = std::move(m_items.front());
		m_items.pop_front();
		return true;
	}

	template<typename It>
	std::size_t try_dequeue_bulk(It first, std::size_t maxCount)
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		std::size_t n = 0;
		while(n < maxCount && !m_items.empty())
		{
			*first = std::move(m_items.front());
			m_items.pop_front();
			++first;
			++n;
		}
		return n;
	}

	std::size_t size_approx() const
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		return m_items.size();
	}

protected:
	mutable std::mutex m_mutex;
	std::deque<T>      m_items;
};

}// end namespace moodycamel
