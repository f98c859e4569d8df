// dvm:: exception hierarchy of the drop-in host library.  Same class names and
// constructors as the reference's src/Exceptions.hpp:13-81, so code written
// against the reference catches the same types; status codes of the C ABI are
// mapped onto them by dvm::check_status.
#ifndef DVMPP_B200_EXCEPTIONS_HPP
#define DVMPP_B200_EXCEPTIONS_HPP

#include <stdexcept>
#include <string>

namespace dvm {

class DVMException : public std::runtime_error {
  public:
    explicit DVMException(const std::string& m) : std::runtime_error(m) {}
    explicit DVMException(const char* m) : std::runtime_error(m) {}
};

class SizeMismatchException : public DVMException {
  public:
    explicit SizeMismatchException(const std::string& where)
        : DVMException("Size mismatch in " + where) {}
};

class FileIOException : public DVMException {
  public:
    explicit FileIOException(const std::string& m) : DVMException(m) {}
    static FileIOException cannotOpen(const std::string& f) {
        return FileIOException("Cannot open file: " + f);
    }
    static FileIOException cannotWrite(const std::string& f) {
        return FileIOException("Cannot write to file: " + f);
    }
    static FileIOException cannotRead(const std::string& f) {
        return FileIOException("Cannot read file: " + f);
    }
};

class XMLParseException : public DVMException {
  public:
    explicit XMLParseException(const std::string& m) : DVMException(m) {}
    static XMLParseException cannotLoad(const std::string& f, const std::string& why) {
        return XMLParseException("Cannot load XML file '" + f + "': " + why);
    }
    static XMLParseException missingParameter(const std::string& level, const std::string& p) {
        return XMLParseException("Missing XML parameter: <" + level + "><" + p + ">");
    }
    static XMLParseException invalidOption(const std::string& level, const std::string& p,
                                           const std::string& options) {
        return XMLParseException("Invalid option for <" + level + "><" + p +
                                 ">. Valid options: " + options);
    }
};

class AlgorithmException : public DVMException {
  public:
    explicit AlgorithmException(const std::string& m) : DVMException(m) {}
};

class VortexException : public DVMException {
  public:
    explicit VortexException(const std::string& m) : DVMException(m) {}
};

// Throws the dvm:: exception matching a C-ABI status (no-op for DVM_OK).
void check_status(int status, const char* where);

}  // namespace dvm

#endif
