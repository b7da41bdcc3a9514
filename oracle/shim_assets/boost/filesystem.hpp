/* Stand-in for the one use of boost::filesystem in the reference's OBJ parser
 * (src/parsers/obj_parser.cpp:250-262): path(obj).parent_path() / mtllib, then native().
 * Boost is not installed; this covers plain relative and absolute POSIX file names. */
#pragma once
#include <string>

namespace boost {
namespace filesystem {

class path {
public:
    path() = default;
    path(const std::string& s) : s_(s) {}
    path(const char* s) : s_(s) {}
    path parent_path() const {
        const std::string::size_type i = s_.find_last_of('/');
        if (i == std::string::npos) return path();
        return path(i == 0 ? std::string("/") : s_.substr(0, i));
    }
    const std::string& native() const { return s_; }

private:
    std::string s_;
};

inline path operator/(const path& a, const path& b) {
    if (a.native().empty()) return b;
    if (!a.native().empty() && a.native().back() == '/') return path(a.native() + b.native());
    return path(a.native() + "/" + b.native());
}

}  // namespace filesystem
}  // namespace boost
