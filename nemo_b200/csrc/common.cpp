#include "common.hpp"

#include <cuda_runtime_api.h>

#include <sstream>

namespace nemo_b200 {

void
fail(int code, const std::string& msg)
{
	throw Exception(code, msg);
}

void
cudaCheck(int err, const char* what, const char* file, int line)
{
	if(err == 0) {
		return;
	}
	cudaError_t e = cudaError_t(err);
	std::ostringstream msg;
	msg << "CUDA error " << err << " (" << cudaGetErrorString(e) << ") in " << what
		<< " at " << file << ":" << line;
	int code = (e == cudaErrorMemoryAllocation) ? NEMO_CUDA_MEMORY_ERROR : NEMO_CUDA_INVOCATION_ERROR;
	throw Exception(code, msg.str());
}

} // namespace nemo_b200
