// Reference CPU render driver (test infrastructure: the oracle and the CPU baseline).
//
// Renders one SDL scene through the reference's own C API, mirroring the call sequence of
// PhotonCLI (PhotonCLI/Source/CliStaticImageRenderer.cpp:21-140):
//   phInit -> phCreateEngine(id, threads) -> phSetWorkingDirectory -> phLoadCommands
//   -> phUpdate -> [timed] phRender -> phCreateFrame -> phAquireFrameRaw -> raw RGB out.
// Only phRender is timed (scene parse and BVH build are reported separately), as the
// CPU baseline plan requires.
//
// Usage: ph_ref_render <scene.p2> <threads> <max-bounces> <out.rgbf32>
// Writes the raw developed frame (float32 RGB, row-major, origin lower-left as the reference
// stores it) and prints one JSON line with timings to stdout.
#include <ph_c_core.h>

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

	const auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
	std::printf(
		"{\"width\": %u, \"height\": %u, \"threads\": %u, \"max_bounces\": %u, "
		"\"load_s\": %.6f, \"update_s\": %.6f, \"render_s\": %.6f}\n",
		w, h, threads, maxBounces, sec(t0, t1), sec(t1, t2), sec(t2, t3));

	phDeleteFrame(frameId);
	phDeleteEngine(engineId);
	phExit();
	return 0;
}
