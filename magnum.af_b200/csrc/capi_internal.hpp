// Shared by the translation units that define extern "C" entry points.
#pragma once
#include <functional>

namespace mafb {

// Runs f after checking that a CUDA device is present; exceptions become the
// status codes of include/maf_b200.h and the text returned by maf_last_error().
int capi_run(const std::function<void()>& f);

// Loads the no-allocation mean's module (code and static scratch) in the
// current device's context (noalloc.cu); called when a state is created.
void noalloc_prepare_current_device();

}  // namespace mafb
