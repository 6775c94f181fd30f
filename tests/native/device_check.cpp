// Host-side check of the device rule: an object created with one device current rejects calls
// made with another device current (pg::check_same_device, used by require_same_device).
#include "pg_runtime.h"

#include <cstdio>
#include <cstring>

int main()
{
	pg::check_same_device(0, 0, "geometry 1");
	pg::check_same_device(3, 3, "scene 2");
	try
	{
		pg::check_same_device(0, 1, "geometry 7");
		std::puts("no error for a different device");
		return 1;
	}
	catch(const pg::Error& e)
	{
		if(e.status != pg::PG_ERR_INVALID_ARGUMENT || !std::strstr(e.what(), "geometry 7 lives on device 0") ||
		   !std::strstr(e.what(), "device 1 is current"))
		{
			std::printf("unexpected error: %d %s\n", e.status, e.what());
			return 1;
		}
	}
	std::puts("ok");
	return 0;
}
