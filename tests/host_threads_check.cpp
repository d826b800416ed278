// Prints host_threads() (kron_plan.h): the library's host thread count.
#include "kron_plan.h"

#include <cstdio>

int main()
{
	std::printf("%d\n", dmrgpp::host_threads());
	return 0;
}
