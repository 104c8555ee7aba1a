// ref_shim.h -- force-included when compiling the reference's B.cu for the harness
// (oracle/build_reference.py).  It lets the unmodified source compile with a C++11 library:
// the reference compares std::ifstream objects with NULL (B.cu:3689, 3732, 4514, 4681), which
// needs the pre-C++11 conversion to void*; this overload gives that comparison its meaning
// (the stream failed to open).  Nothing here changes the reference's arithmetic.
#pragma once
#include <fstream>
#include <cstddef>
inline bool operator==(const std::ifstream& f, long) { return !f.is_open(); }
