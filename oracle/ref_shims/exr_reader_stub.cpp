// Oracle build shim (test infrastructure only, never linked into the product).
//
// Engine/Source/DataIO/EXR/ExrFileReader.cpp needs OpenEXR, which is not available here, so that
// TU is left out of the oracle build and this file supplies the class's members instead
// (declared in Engine/Source/DataIO/EXR/ExrFileReader.h). The oracle scenes use PFM images only,
// which the engine reads natively (Engine/Source/DataIO/io_utils.cpp:370); an EXR load throws.
#include "DataIO/EXR/ExrFileReader.h"

#include <stdexcept>

namespace ph
{

ExrFileReader::ExrFileReader(const Path& filePath) :
	m_filePath(filePath)
{}

void ExrFileReader::load(HdrRgbFrame* const out_frame)
{
	loadFromFilesystem(out_frame);
}

void ExrFileReader::loadFromFilesystem(
	HdrRgbFrame*     out_frame,
	std::string_view redChannelName,
	std::string_view greenChannelName,
	std::string_view blueChannelName)
{
	loadStandaloneImageData(m_filePath, out_frame, redChannelName, greenChannelName, blueChannelName);
}

void ExrFileReader::loadStandaloneImageData(
	const Path,
	HdrRgbFrame*,
	std::string_view,
	std::string_view,
	std::string_view)
{
	throw std::runtime_error("EXR input is not available in the oracle build (OpenEXR absent)");
}

}// end namespace ph
