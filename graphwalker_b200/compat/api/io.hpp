// Drop-in GraphWalker API: full-length pread/pwrite helpers
// (the reference's src/api/io.hpp:11-76).
//
// Two deliberate differences in writefile / appendfile:
//  * they write (bufptr - buf) * sizeof(T) bytes, the whole buffer.  The
//    reference passes the element count bufptr - buf as the byte count
//    (io.hpp:62,74), so for sizeof(T) > 1 it writes only the first
//    1/sizeof(T) of the buffer;
//  * writefile opens with O_TRUNC.  The reference opens without it
//    (io.hpp:57), so a shorter write leaves the old file's tail in place.
// No path of this engine reads files written by these helpers; they exist so
// that programs calling them compile, and they write what the call names.
#ifndef DEF_IOUTIL_HPP
#define DEF_IOUTIL_HPP

#include <errno.h>
#include <fcntl.h>
#include <unistd.h>

#include <cassert>
#include <cstdlib>
#include <cstring>
#include <string>

#include "logger/logger.hpp"

template <typename T>
void preada(int f, T* tbuf, size_t nbytes, size_t off = 0) {
  size_t done = 0;
  char* buf = (char*)tbuf;
  while (done < nbytes) {
    ssize_t a = pread(f, buf + done, nbytes - done, off + done);
    if (a <= 0) {
      logstream(LOG_FATAL) << "could not read " << nbytes - done << " bytes: " << strerror(errno) << std::endl;
      return;
    }
    done += (size_t)a;
  }
}

template <typename T>
size_t readfull(int f, T** buf) {
  off_t sz = lseek(f, 0, SEEK_END);
  lseek(f, 0, SEEK_SET);
  *buf = (T*)malloc(sz);
  preada(f, *buf, sz, 0);
  return sz;
}

template <typename T>
void pwritea(int f, T* tbuf, size_t nbytes, size_t off = 0) {
  size_t done = 0;
  const char* buf = (const char*)tbuf;
  while (done < nbytes) {
    ssize_t a = pwrite(f, buf + done, nbytes - done, off + done);
    if (a <= 0) {
      logstream(LOG_FATAL) << "could not write " << nbytes - done << " bytes: " << strerror(errno) << std::endl;
      return;
    }
    done += (size_t)a;
  }
}

template <typename T>
void writefile(std::string fname, T* buf, T*& bufptr) {
  int f = open(fname.c_str(), O_WRONLY | O_CREAT | O_TRUNC, S_IROTH | S_IWOTH | S_IWUSR | S_IRUSR);
  assert(f >= 0);
  pwritea(f, buf, (bufptr - buf) * sizeof(T));
  close(f);
  bufptr = buf;
}

template <typename T>
void appendfile(std::string fname, T* buf, T*& bufptr) {
  int f = open(fname.c_str(), O_WRONLY | O_CREAT | O_APPEND, S_IROTH | S_IWOTH | S_IWUSR | S_IRUSR);
  assert(f >= 0);
  pwritea(f, buf, (bufptr - buf) * sizeof(T));
  close(f);
}

#endif
