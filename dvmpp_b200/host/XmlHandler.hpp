// XML input of the drop-in host library: the reference's XmlHandler interface
// (src/XmlHandler.hpp:15-93) over a small XML reader of our own.
//
// Semantics kept from the reference (src/XmlHandler.cpp): parameters live at
// <DVMpp><level><parameter .../>; every (level, parameter) must be in the option
// map or getNode throws; a missing parameter throws with a hint; string options
// are checked by substring against the allowed list; "val" options marked ">0"
// must be positive.  The option map adds the GPU choices:
//   algorithms/velocity_kernel  direct fmm cuda cuda64
//   algorithms/diffusion_rng    inject philox
#ifndef DVMPP_B200_XMLHANDLER_HPP
#define DVMPP_B200_XMLHANDLER_HPP

#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

namespace dvm {
// One element of the parsed document.
struct XmlNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<std::unique_ptr<XmlNode>> children;
    const XmlNode* child(const std::string& n) const;
    const std::string* attr(const std::string& n) const;
};
// Parses text into a document root (children = top-level elements); throws
// std::runtime_error with a description on malformed input.
std::unique_ptr<XmlNode> parse_xml(const std::string& text);
std::string write_xml(const XmlNode& root);
}  // namespace dvm

class XmlHandler
{
  private:
    std::unique_ptr<dvm::XmlNode> m_doc;
    struct opts {
        std::string level, parameter, attr, info, reqs;
    };
    std::unordered_map<std::string, opts> m_option_map;

    const dvm::XmlNode& getNode(const char* level, const char* parameter) const;
    void check_string(const char* level, const char* parameter, std::string& attr) const;
    void check_value(const char* level, const char* parameter, double attr) const;
    std::string form_key(const char* level, const char* parameter) const;
    void buildOptionMap();

  public:
    XmlHandler();
    XmlHandler(std::string xml_file);
    XmlHandler(const XmlHandler& o);
    XmlHandler& operator=(const XmlHandler& o);

    std::string getStringAttribute(const char* level, const char* parameter,
                                   bool checksep = false) const;
    std::vector<double> getList(const char* level, const char* parameter) const;
    double getValueAttribute(const char* level, const char* parameter) const;
    int getIntAttribute(const char* level, const char* parameter) const;
    bool getBoolAttribute(const char* level, const char* parameter) const;
    // True when <DVMpp><level><parameter> is present (no throw).
    bool has(const char* level, const char* parameter) const;
    void save(std::string filename) const;
    void writeExample(std::string file) const;
};

#endif
