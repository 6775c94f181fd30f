// Oracle build shim (test infrastructure only, never linked into the product).
//
// Blocking variant used by Engine/Source/Utility/Concurrent/TBlockableAtomicQuasiQueue.ipp:13-74
// (adds wait_dequeue and wait_dequeue_bulk). Implemented with a condition variable over the
// mutex-guarded deque of concurrentqueue.h in this directory.
#pragma once

#include "concurrentqueue.h"

#include <condition_variable>

namespace moodycamel
{

template<typename T>
class BlockingConcurrentQueue
{
public:
	BlockingConcurrentQueue() = default;
	explicit BlockingConcurrentQueue(std::size_t /*initialCapacity*/) {}

	BlockingConcurrentQueue(BlockingConcurrentQueue&& other)
	{
		std::lock_guard<std::mutex> lock(other.m_mutex);
		m_items = std::move(other.m_items);
	}

	BlockingConcurrentQueue& operator = (BlockingConcurrentQueue&& other)
	{
		if(this != &other)
		{
			std::scoped_lock lock(m_mutex, other.m_mutex);
			m_items = std::move(other.m_items);
		}
		return *this;
	}

	template<typename U>
	bool enqueue(U&& item)
	{
		{
			std::lock_guard<std::mutex> lock(m_mutex);
			m_items.emplace_back(std::forward<U>(item));
		}
		m_cv.notify_one();
		return true;
	}

	template<typename It>
	bool enqueue_bulk(It first, std::size_t count)
	{
		{
			std::lock_guard<std::mutex> lock(m_mutex);
			for(std::size_t i = 0; i < count; ++i, ++first)
			{
				m_items.emplace_back(*first);
			}
		}
		m_cv.notify_all();
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

	template<typename U>
	void wait_dequeue(U& out)
	{
		std::unique_lock<std::mutex> lock(m_mutex);
		m_cv.wait(lock, [this]{ return !m_items.empty(); });
		out = std::move(m_items.front());
		m_items.pop_front();
	}

	template<typename It>
	std::size_t wait_dequeue_bulk(It first, std::size_t maxCount)
	{
		std::unique_lock<std::mutex> lock(m_mutex);
		m_cv.wait(lock, [this]{ return !m_items.empty(); });
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

private:
	mutable std::mutex      m_mutex;
	std::condition_variable m_cv;
	std::deque<T>           m_items;
};

}// end namespace moodycamel
