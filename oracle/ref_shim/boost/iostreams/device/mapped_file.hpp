// Minimal read-only stand-in for boost::iostreams::mapped_file_source, enough for the
// reference's index builder (ISSLCreateIndex/ISSLCreateIndex.cpp:385-486) and for the
// unused include of its CPU scorer (ISSLScoreOfftargets/ISSLScoreOfftargets.hpp:9).
// Part of the CPU checker's build recipe (oracle/Makefile); never shipped.
#pragma once
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstddef>
#include <stdexcept>
#include <string>

namespace boost {
namespace iostreams {
class mapped_file_source {
   public:
    mapped_file_source() = default;
    ~mapped_file_source() { close(); }
    void open(const std::string& path) {
        close();
        int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error("mapped_file_source: cannot open " + path);
        struct stat st;
        ::fstat(fd, &st);
        size_ = static_cast<std::size_t>(st.st_size);
        // one spare zero page past the end: the builder's run-length loop peeks past EOF
        std::size_t page = static_cast<std::size_t>(::sysconf(_SC_PAGESIZE));
        map_len_ = ((size_ + page - 1) / page + 1) * page;
        void* p = ::mmap(nullptr, map_len_, PROT_READ, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (p == MAP_FAILED) throw std::runtime_error("mapped_file_source: mmap failed");
        if (size_ && ::mmap(p, size_, PROT_READ, MAP_PRIVATE | MAP_FIXED, fd, 0) == MAP_FAILED)
            throw std::runtime_error("mapped_file_source: mmap of file failed");
        ::close(fd);
        data_ = static_cast<const char*>(p);
    }
    void close() {
        if (data_) ::munmap(const_cast<char*>(data_), map_len_);
        data_ = nullptr;
        size_ = map_len_ = 0;
    }
    const char* data() const { return data_; }
    std::size_t size() const { return size_; }
    const char* begin() const { return data_; }
    const char* end() const { return data_ + size_; }

   private:
    const char* data_ = nullptr;
    std::size_t size_ = 0, map_len_ = 0;
};
}  // namespace iostreams
}  // namespace boost
