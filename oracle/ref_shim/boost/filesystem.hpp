// Minimal stand-in for the three boost::filesystem calls the reference solver
// makes (exists, create_directory, create_directories).  Written for this
// project so the read-only reference sources can be compiled without Boost;
// it is used only by oracle/Makefile.ref to build the parity checker.
#pragma once
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <cerrno>

namespace boost {
namespace filesystem {

inline bool exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

inline bool create_directory(const std::string& p) {
    return ::mkdir(p.c_str(), 0755) == 0;
}

inline bool create_directories(const std::string& p) {
    if (p.empty()) return false;
    std::string cur;
    bool made = false;
    for (std::size_t i = 0; i <= p.size(); ++i) {
        if (i == p.size() || p[i] == '/') {
            if (!cur.empty() && !exists(cur)) made = create_directory(cur) || made;
        }
        if (i < p.size()) cur.push_back(p[i]);
    }
    return made;
}

}  // namespace filesystem
}  // namespace boost
