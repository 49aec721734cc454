// cvl_internal.h -- what the host-side translation units of libcvl share
// beyond the public C ABI.
#pragma once

#include <string>

// Records msg as the calling thread's cvl_last_error() and returns code.
int cvl_fail(int code, const std::string &msg);
