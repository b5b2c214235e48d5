// gwfa_internal.h — declarations shared by the host-side translation units of libgwfa_b200.
#pragma once
#include <cstdint>

// Thread-local last-error message (gwf_last_error).
void gwf_set_error(const char *msg);
void gwf_set_errorf(const char *fmt, ...);
