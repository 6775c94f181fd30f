// Compressed 8-wide BVH builder: binned SAH binary tree, greedy collapse to 8-wide nodes,
// octant slot assignment and conservative 8-bit child-box quantization.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <stdexcept>
#include <thread>

namespace pg
{
namespace
{

struct Box
{
	float lo[3] = { std::numeric_limits<float>::infinity(),  std::numeric_limits<float>::infinity(),
	                std::numeric_limits<float>::infinity()};
	float hi[3] = {-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
	               -std::numeric_limits<float>::infinity()};

	void grow(const Box& b)
	{
		for(int a = 0; a < 3; ++a)
		{
			lo[a] = std::min(lo[a], b.lo[a]);
			hi[a] = std::max(hi[a], b.hi[a]);
		}
	}
	void grow(const float* p)
	{
		for(int a = 0; a < 3; ++a)
		{
			lo[a] = std::min(lo[a], p[a]);
			hi[a] = std::max(hi[a], p[a]);
		}
	}
	bool valid() const { return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2]; }
	float area() const
	{
		if(!valid())
		{
			return 0.0f;
		}
		const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
		return 2.0f * (dx * dy + dy * dz + dz * dx);
	}
};

struct BinNode
{
	Box      box;
	int32_t  left = -1;   // -1 for a leaf
	int32_t  right = -1;
	uint32_t begin = 0;
	uint32_t count = 0;
};

constexpr int kBins = 32;
constexpr uint32_t kMaxLeafTris = 3;   // the node layout's limit (unary leaf counts of 1..3)
constexpr std::size_t kParallelThreshold = 1u << 15;

struct BinaryBuilder
{
	const Box*            prim_boxes;
	const float*          centroids;      // [n][3]
	uint32_t              max_leaf = kMaxLeafTris;
	std::vector<uint32_t> indices;
	std::vector<BinNode>  nodes;
	std::atomic<int32_t>  next_node{0};
	std::atomic<int>      max_depth{0};
	std::atomic<int>      live_tasks{0};
	int                   max_tasks = 1;

	int32_t alloc_node()
	{
		return next_node.fetch_add(1, std::memory_order_relaxed);
	}

	void note_depth(int d)
	{
		int cur = max_depth.load(std::memory_order_relaxed);
		while(d > cur && !max_depth.compare_exchange_weak(cur, d, std::memory_order_relaxed))
		{}
	}

	void build(int32_t node_index, uint32_t begin, uint32_t end, int depth)
	{
		BinNode& node = nodes[node_index];
		node.begin = begin;
		node.count = end - begin;
		Box box, cbox;
		for(uint32_t i = begin; i < end; ++i)
		{
			const uint32_t p = indices[i];
			box.grow(prim_boxes[p]);
			cbox.grow(&centroids[3 * p]);
		}
		node.box = box;
		note_depth(depth);

		const uint32_t n = end - begin;
		if(n <= max_leaf)
		{
			return;
		}

		// Binned SAH over all three axes.
		int best_axis = -1;
		int best_split = -1;
		float best_cost = std::numeric_limits<float>::infinity();
		for(int axis = 0; axis < 3; ++axis)
		{
			const float extent = cbox.hi[axis] - cbox.lo[axis];
			if(!(extent > 0.0f))
			{
				continue;
			}
			Box bin_box[kBins];
			uint32_t bin_count[kBins] = {};
			const float scale = kBins / extent;
			for(uint32_t i = begin; i < end; ++i)
			{
				const uint32_t p = indices[i];
				int b = static_cast<int>((centroids[3 * p + axis] - cbox.lo[axis]) * scale);
				b = std::min(std::max(b, 0), kBins - 1);
				bin_box[b].grow(prim_boxes[p]);
				++bin_count[b];
			}
			float right_area[kBins];
			uint32_t right_count[kBins];
			Box acc;
			uint32_t cnt = 0;
			for(int b = kBins - 1; b > 0; --b)
			{
				acc.grow(bin_box[b]);
				cnt += bin_count[b];
				right_area[b] = acc.area();
				right_count[b] = cnt;
			}
			acc = Box{};
			cnt = 0;
			for(int b = 0; b < kBins - 1; ++b)
			{
				acc.grow(bin_box[b]);
				cnt += bin_count[b];
				if(cnt == 0 || right_count[b + 1] == 0)
				{
					continue;
				}
				const float cost = acc.area() * cnt + right_area[b + 1] * right_count[b + 1];
				if(cost < best_cost)
				{
					best_cost = cost;
					best_axis = axis;
					best_split = b;
				}
			}
		}

		uint32_t mid;
		if(best_axis >= 0)
		{
			const float extent = cbox.hi[best_axis] - cbox.lo[best_axis];
			const float scale = kBins / extent;
			const float lo = cbox.lo[best_axis];
			const int split = best_split;
			const int axis = best_axis;
			auto it = std::partition(indices.begin() + begin, indices.begin() + end,
				[&](uint32_t p)
				{
					int b = static_cast<int>((centroids[3 * p + axis] - lo) * scale);
					b = std::min(std::max(b, 0), kBins - 1);
					return b <= split;
				});
			mid = static_cast<uint32_t>(it - indices.begin());
			if(mid == begin || mid == end)
			{
				mid = begin + n / 2;
			}
		}
		else
		{
			// All centroids coincide: split by index.
			mid = begin + n / 2;
		}

		const int32_t l = alloc_node();
		const int32_t r = alloc_node();
		node.left = l;
		node.right = r;

		const bool big = (mid - begin) >= kParallelThreshold && (end - mid) >= kParallelThreshold;
		if(big && live_tasks.fetch_add(1) < max_tasks)
		{
			auto fut = std::async(std::launch::async, [&, l, begin, mid, depth]
			{
				build(l, begin, mid, depth + 1);
			});
			build(r, mid, end, depth + 1);
			fut.get();
			live_tasks.fetch_sub(1);
		}
		else
		{
			if(big)
			{
				live_tasks.fetch_sub(1);
			}
			build(l, begin, mid, depth + 1);
			build(r, mid, end, depth + 1);
		}
	}
};

struct WideCollapser
{
	const BinaryBuilder& bin;
	const float*         tris;
	const uint32_t*      materials;
	const uint32_t*      emitters;
	float                pad;
	std::vector<WideNode> nodes;
	std::vector<LeafTri>  leaf_tris;
	int                   max_depth = 0;

	struct Pending
	{
		int32_t bin_node;
		uint32_t wide_index;
		int depth;
	};

	static void set_byte(WideNode& n, int word, int byte, uint32_t value)
	{
		n.w[word] = (n.w[word] & ~(0xFFu << (8 * byte))) | ((value & 0xFFu) << (8 * byte));
	}

	Box padded(const Box& b) const
	{
		Box r = b;
		for(int a = 0; a < 3; ++a)
		{
			r.lo[a] = b.lo[a] - pad;
			r.hi[a] = b.hi[a] + pad;
		}
		return r;
	}

	void append_leaf_tris(const BinNode& leaf)
	{
		for(uint32_t i = 0; i < leaf.count; ++i)
		{
			const uint32_t p = bin.indices[leaf.begin + i];
			const float* v = tris + 9 * static_cast<std::size_t>(p);
			LeafTri t;
			t.v0x = v[0]; t.v0y = v[1]; t.v0z = v[2]; t.prim = p;
			t.v1x = v[3]; t.v1y = v[4]; t.v1z = v[5]; t.material = materials ? materials[p] : 0u;
			t.v2x = v[6]; t.v2y = v[7]; t.v2z = v[8]; t.emitter_plus_one = emitters ? emitters[p] : 0u;
			leaf_tris.push_back(t);
		}
	}

	void run()
	{
		nodes.emplace_back();
		std::memset(&nodes[0], 0, sizeof(WideNode));
		std::vector<Pending> queue;
		queue.push_back({0, 0u, 1});
		std::size_t head = 0;
		while(head < queue.size())
		{
			const Pending job = queue[head++];
			max_depth = std::max(max_depth, job.depth);

			// Gather up to 8 children by repeatedly opening the largest internal child.
			std::vector<int32_t> children;
			const BinNode& root = bin.nodes[job.bin_node];
			if(root.left < 0)
			{
				children.push_back(job.bin_node);   // a lone leaf (tiny scenes)
			}
			else
			{
				children.push_back(root.left);
				children.push_back(root.right);
			}
			while(children.size() < 8)
			{
				int best = -1;
				float best_area = -1.0f;
				for(int i = 0; i < static_cast<int>(children.size()); ++i)
				{
					const BinNode& c = bin.nodes[children[i]];
					if(c.left >= 0 && c.box.area() > best_area)
					{
						best_area = c.box.area();
						best = i;
					}
				}
				if(best < 0)
				{
					break;
				}
				const BinNode& c = bin.nodes[children[best]];
				children[best] = c.left;
				children.push_back(c.right);
			}

			// Octant slot assignment: slot bit a set <=> child centroid on the negative side of
			// the parent's centroid along axis a; resolved greedily by best alignment.
			Box parent_box;
			for(int32_t c : children)
			{
				parent_box.grow(bin.nodes[c].box);
			}
			float pc[3];
			for(int a = 0; a < 3; ++a)
			{
				pc[a] = 0.5f * (parent_box.lo[a] + parent_box.hi[a]);
			}
			int slot_of[8];
			bool slot_used[8] = {};
			bool child_done[8] = {};
			const int k = static_cast<int>(children.size());
			for(int round = 0; round < k; ++round)
			{
				float best_score = -std::numeric_limits<float>::infinity();
				int bc = -1, bs = -1;
				for(int c = 0; c < k; ++c)
				{
					if(child_done[c])
					{
						continue;
					}
					const Box& b = bin.nodes[children[c]].box;
					float d[3];
					for(int a = 0; a < 3; ++a)
					{
						d[a] = 0.5f * (b.lo[a] + b.hi[a]) - pc[a];
					}
					for(int s = 0; s < 8; ++s)
					{
						if(slot_used[s])
						{
							continue;
						}
						float score = 0.0f;
						for(int a = 0; a < 3; ++a)
						{
							score += ((s >> a) & 1) ? -d[a] : d[a];
						}
						if(score > best_score)
						{
							best_score = score;
							bc = c;
							bs = s;
						}
					}
				}
				child_done[bc] = true;
				slot_used[bs] = true;
				slot_of[bc] = bs;
			}

			// Quantization frame of this node.
			Box qbox;
			Box cbox[8];
			for(int c = 0; c < k; ++c)
			{
				cbox[c] = padded(bin.nodes[children[c]].box);
				qbox.grow(cbox[c]);
			}
			WideNode node;
			std::memset(&node, 0, sizeof(node));
			float p[3];
			int e[3];
			float scale[3];
			for(int a = 0; a < 3; ++a)
			{
				p[a] = qbox.lo[a];
				const float extent = qbox.hi[a] - qbox.lo[a];
				// 254 quanta cover the extent, one spare quantum absorbs the rounding of p + q*s.
				int ex = extent > 0.0f
					? static_cast<int>(std::ceil(std::log2(static_cast<double>(extent) / 254.0)))
					: -126;
				ex = std::min(std::max(ex, -126), 127);
				while(std::ldexp(254.0, ex) < static_cast<double>(extent) && ex < 127)
				{
					++ex;
				}
				e[a] = ex;
				scale[a] = std::ldexp(1.0f, ex);
			}
			std::memcpy(&node.w[0], &p[0], 4);
			std::memcpy(&node.w[1], &p[1], 4);
			std::memcpy(&node.w[2], &p[2], 4);

			// Children: internal ones allocated contiguously in slot order, leaves' triangles
			// appended contiguously.
			int child_at_slot[8];
			for(int s = 0; s < 8; ++s)
			{
				child_at_slot[s] = -1;
			}
			for(int c = 0; c < k; ++c)
			{
				child_at_slot[slot_of[c]] = c;
			}
			uint32_t imask = 0;
			int num_internal = 0;
			for(int s = 0; s < 8; ++s)
			{
				const int c = child_at_slot[s];
				if(c >= 0 && bin.nodes[children[c]].left >= 0)
				{
					imask |= 1u << s;
					++num_internal;
				}
			}
			const uint32_t child_base = static_cast<uint32_t>(nodes.size());
			const uint32_t tri_base = static_cast<uint32_t>(leaf_tris.size());
			node.w[3] = static_cast<uint32_t>(e[0] + 127) | (static_cast<uint32_t>(e[1] + 127) << 8) |
			            (static_cast<uint32_t>(e[2] + 127) << 16) | (imask << 24);
			node.w[4] = child_base;
			node.w[5] = tri_base;
			nodes.resize(nodes.size() + num_internal);

			int internal_rank = 0;
			uint32_t tri_offset = 0;
			for(int s = 0; s < 8; ++s)
			{
				const int c = child_at_slot[s];
				if(c < 0)
				{
					continue;
				}
				const BinNode& child = bin.nodes[children[c]];
				uint32_t meta;
				if(child.left >= 0)
				{
					meta = (1u << 5) | (24u + static_cast<uint32_t>(s));
					queue.push_back({children[c], child_base + internal_rank, job.depth + 1});
					++internal_rank;
				}
				else
				{
					const uint32_t unary = (1u << child.count) - 1u;
					meta = (unary << 5) | tri_offset;
					tri_offset += child.count;
					append_leaf_tris(child);
				}
				set_byte(node, 6 + s / 4, s % 4, meta);

				// Conservative quantization, verified in FP32 exactly as the traversal decodes.
				for(int a = 0; a < 3; ++a)
				{
					long qlo = static_cast<long>(std::floor((cbox[c].lo[a] - p[a]) / scale[a]));
					long qhi = static_cast<long>(std::ceil((cbox[c].hi[a] - p[a]) / scale[a]));
					qlo = std::max(0L, std::min(255L, qlo));
					qhi = std::max(0L, std::min(255L, qhi));
					while(qlo > 0 && p[a] + static_cast<float>(qlo) * scale[a] > cbox[c].lo[a])
					{
						--qlo;
					}
					while(qhi < 255 && p[a] + static_cast<float>(qhi) * scale[a] < cbox[c].hi[a])
					{
						++qhi;
					}
					// words: qlo.x 8,9  qlo.y 10,11  qlo.z 12,13  qhi.x 14,15  qhi.y 16,17  qhi.z 18,19
					set_byte(node, 8 + 2 * a + s / 4, s % 4, static_cast<uint32_t>(qlo));
					set_byte(node, 14 + 2 * a + s / 4, s % 4, static_cast<uint32_t>(qhi));
				}
			}
			nodes[job.wide_index] = node;
		}
	}
};

}// end anonymous namespace

WideBvh build_wide_bvh(const BvhBuildInput& in)
{
	const auto t0 = std::chrono::steady_clock::now();
	if(!in.tris || in.num_tris == 0)
	{
		throw std::runtime_error("build_wide_bvh: no triangles");
	}
	if(in.num_tris > 0xFFFFFFF0ull)
	{
		throw std::runtime_error("build_wide_bvh: too many triangles");
	}
	const std::size_t n = in.num_tris;

	std::vector<Box> boxes(n);
	std::vector<float> centroids(3 * n);
	float max_abs = std::max(in.max_origin_abs, 1.0f);
	for(std::size_t i = 0; i < n; ++i)
	{
		const float* v = in.tris + 9 * i;
		Box b;
		b.grow(v);
		b.grow(v + 3);
		b.grow(v + 6);
		for(int a = 0; a < 3; ++a)
		{
			if(!std::isfinite(b.lo[a]) || !std::isfinite(b.hi[a]))
			{
				// Non-finite vertices: give the triangle an empty-but-valid box at the origin;
				// the watertight test rejects it anyway.
				b.lo[a] = 0.0f;
				b.hi[a] = 0.0f;
			}
			max_abs = std::max(max_abs, std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
		}
		boxes[i] = b;
		for(int a = 0; a < 3; ++a)
		{
			centroids[3 * i + a] = 0.5f * (b.lo[a] + b.hi[a]);
		}
	}

	if(in.max_leaf_tris < 1 || in.max_leaf_tris > kMaxLeafTris)
	{
		throw std::runtime_error("build_wide_bvh: max_leaf_tris must be 1, 2 or 3");
	}
	BinaryBuilder bb;
	bb.max_leaf = in.max_leaf_tris;
	bb.prim_boxes = boxes.data();
	bb.centroids = centroids.data();
	bb.indices.resize(n);
	for(std::size_t i = 0; i < n; ++i)
	{
		bb.indices[i] = static_cast<uint32_t>(i);
	}
	bb.nodes.resize(2 * n + 1);
	bb.max_tasks = std::max(1u, std::thread::hardware_concurrency()) * 2;
	const int32_t root = bb.alloc_node();
	bb.build(root, 0, static_cast<uint32_t>(n), 1);
	bb.nodes.resize(bb.next_node.load());

	WideCollapser wc{bb, in.tris, in.materials, in.emitters, 4.0e-6f * max_abs};
	wc.leaf_tris.reserve(n);
	wc.run();

	WideBvh out;
	out.nodes = std::move(wc.nodes);
	out.tris = std::move(wc.leaf_tris);
	out.stats.num_nodes = out.nodes.size();
	out.stats.num_leaf_tris = out.tris.size();
	out.stats.max_depth = wc.max_depth;
	out.stats.binary_max_depth = bb.max_depth.load();
	out.stats.box_padding = wc.pad;
	out.stats.build_seconds =
		std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	if(out.stats.max_depth >= kTraversalStackSize)
	{
		throw std::runtime_error("build_wide_bvh: tree deeper than the traversal stack");
	}
	return out;
}

}// end namespace pg
