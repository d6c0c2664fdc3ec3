/*
 * Stand-in for the one boost::filesystem use of the reference's hot-path
 * sources: path(...).filename().string().  Oracle build scaffolding only.
 */
#ifndef ORACLE_STUB_BOOST_FILESYSTEM_HPP
#define ORACLE_STUB_BOOST_FILESYSTEM_HPP
#include <string>
namespace boost {
namespace filesystem {
class path {
public:
    path(const std::string& s) : s_(s) {}
    path(const char* s) : s_(s) {}
    path filename() const {
        std::string::size_type k = s_.find_last_of('/');
        return path(k == std::string::npos ? s_ : s_.substr(k + 1));
    }
    std::string string() const { return s_; }
private:
    std::string s_;
};
}  // namespace filesystem
}  // namespace boost
#endif
