// Test stub: the part of OpenMM's OpenMMException the adapter uses.
#pragma once
#include <exception>
#include <string>
namespace OpenMM {
class OpenMMException : public std::exception {
public:
    explicit OpenMMException(const std::string& message) : message_(message) {}
    const char* what() const noexcept override { return message_.c_str(); }
private:
    std::string message_;
};
}  // namespace OpenMM
