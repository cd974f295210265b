// Drop-in GraphWalker API: basic types and constants.
// Same names and widths as the reference's src/api/datatype.hpp:8-23 so that
// programs written against it compile unchanged.
#ifndef GW_COMPAT_DATATYPE_HPP
#define GW_COMPAT_DATATYPE_HPP

#include <stdint.h>

#include <cstdlib>
#include <vector>

#include "logger/logger.hpp"

#ifndef RAND_MAX
#define RAND_MAX 2147483647
#endif
#define FILE_SIZE 1024                         // GB per CSR file (one file)
#define VERT_SIZE 64 * 1024 * 1024             // preprocessing buffer, vertices
#define EDGE_SIZE 256 * 1024 * 1024            // preprocessing buffer, edges
#define WALK_BUFFER_SIZE 4 * 1024              // walks per host walk buffer
#define MEM_BUDGET 44 * 1024 * 1024            // KB, for compNmblocks

typedef uint32_t vid_t;   // vertex id
typedef uint64_t eid_t;   // edge offset
typedef uint64_t wid_t;   // walk count / id
typedef uint32_t bid_t;   // block id
typedef uint16_t hid_t;   // hop
typedef uint8_t tid_t;    // thread id
typedef unsigned VertexDataType;
typedef unsigned long WalkDataType;  // the 64-bit (source, current, hop) walk

#endif
