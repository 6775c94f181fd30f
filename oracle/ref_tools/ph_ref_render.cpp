// Reference CPU render driver (test infrastructure: the oracle and the CPU baseline).
//
// Renders one SDL scene through the reference's own C API, mirroring the call sequence of
// PhotonCLI (PhotonCLI/Source/CliStaticImageRenderer.cpp:21-140):
//   phInit -> phCreateEngine(id, threads) -> phSetWorkingDirectory -> phLoadCommands
//   -> phUpdate -> [timed] phRender -> phCreateFrame -> phAquireFrameRaw -> raw RGB out.
// Only phRender is timed (scene parse and BVH build are reported separately), as the
// CPU baseline plan requires.
//
// Usage: ph_ref_render <scene.p2> <threads> <max-bounces> <out.rgbf32> [repeats]
// Writes the raw developed frame (float32 RGB, row-major, origin lower-left as the reference
// stores it) and prints one JSON line with timings to stdout per repeat. Each repeat runs
// phUpdate (untimed) and phRender (timed) on the already loaded scene.
#include <ph_c_core.h>

#include <algorithm>
#include <chrono>
#include <filesystem>
#include <cstdio>
#include <cstdlib>
#include <string>

extern "C" unsigned int ph_oracle_max_ray_bounces;

int main(int argc, char** argv)
{
	if(argc < 5)
	{
		std::fprintf(stderr, "usage: %s <scene.p2> <threads> <max-bounces> <out.rgbf32>\n", argv[0]);
		return 2;
	}
	const std::string scenePath = argv[1];
	const unsigned threads = static_cast<unsigned>(std::atoi(argv[2]));
	const unsigned maxBounces = static_cast<unsigned>(std::atoi(argv[3]));
	const std::string outPath = argv[4];
	const int repeats = argc >= 6 ? std::max(1, std::atoi(argv[5])) : 1;

	ph_oracle_max_ray_bounces = maxBounces;

	// The engine reads (and on first use writes) ./Config/EngineConfig.ini during phInit
	// (Engine/Source/Api/EngineInitSettings.cpp:13-24); make sure the folder exists.
	std::filesystem::create_directories("Config");

	using Clock = std::chrono::steady_clock;
	if(!phInit())
	{
		std::fprintf(stderr, "phInit failed\n");
		return 1;
	}

	PhUInt64 engineId = 0;
	phCreateEngine(&engineId, threads);

	const auto slash = scenePath.find_last_of('/');
	const std::string workDir = slash == std::string::npos ? "." : scenePath.substr(0, slash);
	phSetWorkingDirectory(engineId, workDir.c_str());

	const auto t0 = Clock::now();
	if(!phLoadCommands(engineId, scenePath.c_str()))
	{
		std::fprintf(stderr, "phLoadCommands failed for %s\n", scenePath.c_str());
		return 1;
	}
	const auto t1 = Clock::now();
	const auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
	for(int rep = 0; rep < repeats; ++rep)
	{
		const auto t2a = Clock::now();
		phUpdate(engineId);
		const auto t2 = Clock::now();
		phRender(engineId);
		const auto t3 = Clock::now();

		PhUInt32 w = 0, h = 0;
		phGetRenderDimension(engineId, &w, &h);
		PhUInt64 frameId = 0;
		phCreateFrame(&frameId, w, h);
		phAquireFrameRaw(engineId, 0, frameId);
		const PhFloat32* data = nullptr;
		phGetFrameRgbData(frameId, &data);

		FILE* f = std::fopen(outPath.c_str(), "wb");
		if(!f || !data)
		{
			std::fprintf(stderr, "cannot write %s\n", outPath.c_str());
			return 1;
		}
		std::fwrite(data, sizeof(float), static_cast<std::size_t>(w) * h * 3, f);
		std::fclose(f);

		std::printf(
			"{\"width\": %u, \"height\": %u, \"threads\": %u, \"max_bounces\": %u, \"repeat\": %d, "
			"\"load_s\": %.6f, \"update_s\": %.6f, \"render_s\": %.6f}\n",
			w, h, threads, maxBounces, rep, sec(t0, t1), sec(t2a, t2), sec(t2, t3));
		std::fflush(stdout);
		phDeleteFrame(frameId);
	}

	phDeleteEngine(engineId);
	phExit();
	return 0;
}
