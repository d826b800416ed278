// Prints host_threads() and validation_requested() (kron_plan.h): the
// library's host thread count and whether its debug-mode check is on.
#include "kron_plan.h"

#include <cstdio>

int main()
{
	std::printf("%d %d\n", dmrgpp::host_threads(), dmrgpp::validation_requested() ? 1 : 0);
	return 0;
}
