// Field-file writer shared by the C-ABI entry points (mplb_io.cu) and the
// write-step snapshot's writer thread (mplb_gpu.cu).  Returns 0 or an MPLB_E_*
// code with the message in *err; touches no thread-local error state, so it
// can run on any thread.
#pragma once
#include <cstdint>
#include <string>

int mplb_io_write(const char* root, int32_t pid, uint32_t time, int32_t format, const char* name,
                  const double* field, uint64_t n, uint32_t vsize, bool scalar, std::string* err);
