// gwfa_internal.h — declarations shared by the host-side translation units of libgwfa_b200.
#pragma once
#include <cstddef>
#include <cstdint>

// Thread-local last-error message (gwf_last_error).
void gwf_set_error(const char *msg);
void gwf_set_errorf(const char *fmt, ...);

// The whole file, decompressed when it is gzip ("-" or NULL: standard input), in a malloc'd
// buffer of *len bytes; NULL with the error set on failure.
char *gwf_read_file(const char *path, size_t *len);

// IUPAC complement of a base, upper and lower case; other bytes map to themselves (U -> A).
unsigned char gwf_comp_base(unsigned char c);
