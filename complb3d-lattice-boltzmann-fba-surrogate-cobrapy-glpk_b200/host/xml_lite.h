// xml_lite.h -- the small XML reader the host driver needs for CompLaB.xml:
// elements, text, comments, the <?xml ... ?> declaration; attributes are
// skipped (the CompLaB schema has none).  Lookup mirrors Palabos XMLreader's
// doc["parameters"]["chemistry"]["substrate0"]["name_of_substrates"].read(v)
// used by initialize_complab (src/complab_functions.hh:621-1349): a missing
// element throws XmlMissing, which callers turn into the reference's default.
#pragma once
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace clhost {

struct XmlMissing : std::runtime_error {
    explicit XmlMissing(const std::string& path) : std::runtime_error("missing XML element: " + path) {}
};

struct XmlNode {
    std::string name, text, path;
    std::vector<std::unique_ptr<XmlNode>> kids;

    const XmlNode* find(const std::string& n) const {
        for (const auto& k : kids) if (k->name == n) return k.get();
        return nullptr;
    }
    const XmlNode& operator[](const std::string& n) const {
        const XmlNode* k = find(n);
        if (!k) throw XmlMissing(path + "/" + n);
        return *k;
    }
    bool has(const std::string& n) const { return find(n) != nullptr; }

    std::string str() const {
        size_t a = 0, b = text.size();
        while (a < b && std::isspace((unsigned char)text[a])) ++a;
        while (b > a && std::isspace((unsigned char)text[b - 1])) --b;
        return text.substr(a, b - a);
    }
    double num() const {
        const std::string s = str();
        char* end = nullptr;
        const double v = std::strtod(s.c_str(), &end);
        if (s.empty() || (end && *end)) throw std::runtime_error("not a number at " + path + ": '" + s + "'");
        return v;
    }
    long integer() const { return (long)num(); }
    // true/yes/1/on (any case) as the reference's readers accept
    bool flag() const {
        std::string s = str();
        for (auto& c : s) c = (char)std::tolower((unsigned char)c);
        return s == "true" || s == "yes" || s == "1" || s == "on";
    }
    // whitespace-separated list of numbers (e.g. <pore>2 3</pore>)
    std::vector<double> nums() const {
        std::istringstream is(str());
        std::vector<double> v;
        double d;
        while (is >> d) v.push_back(d);
        return v;
    }
    std::vector<std::string> words() const {
        std::istringstream is(str());
        std::vector<std::string> v;
        std::string w;
        while (is >> w) v.push_back(w);
        return v;
    }
};

class XmlDoc {
public:
    explicit XmlDoc(const std::string& file) {
        std::ifstream f(file);
        if (!f) throw std::runtime_error("cannot open " + file);
        std::stringstream ss;
        ss << f.rdbuf();
        src_ = ss.str();
        root_.name = "";
        root_.path = "";
        parse_children(root_);
    }
    const XmlNode& root() const { return root_; }
    const XmlNode& operator[](const std::string& n) const { return root_[n]; }

private:
    std::string src_;
    size_t pos_ = 0;
    XmlNode root_;

    [[noreturn]] void fail(const std::string& what) const {
        throw std::runtime_error("XML parse error at byte " + std::to_string(pos_) + ": " + what);
    }
    bool starts(const char* s) const { return src_.compare(pos_, std::char_traits<char>::length(s), s) == 0; }
    void skip_to(const char* s) {
        const size_t p = src_.find(s, pos_);
        if (p == std::string::npos) fail(std::string("unterminated, expected ") + s);
        pos_ = p + std::char_traits<char>::length(s);
    }

    // parse children of `parent` until its closing tag (or end of input for the root)
    void parse_children(XmlNode& parent) {
        while (pos_ < src_.size()) {
            if (src_[pos_] != '<') {
                const size_t p = src_.find('<', pos_);
                parent.text += src_.substr(pos_, (p == std::string::npos ? src_.size() : p) - pos_);
                pos_ = (p == std::string::npos) ? src_.size() : p;
                continue;
            }
            if (starts("<!--")) { skip_to("-->"); continue; }
            if (starts("<?")) { skip_to("?>"); continue; }
            if (starts("<![CDATA[")) {
                pos_ += 9;
                const size_t p = src_.find("]]>", pos_);
                if (p == std::string::npos) fail("unterminated CDATA");
                parent.text += src_.substr(pos_, p - pos_);
                pos_ = p + 3;
                continue;
            }
            if (starts("<!")) { skip_to(">"); continue; }
            if (starts("</")) {
                pos_ += 2;
                size_t p = pos_;
                while (p < src_.size() && src_[p] != '>' && !std::isspace((unsigned char)src_[p])) ++p;
                const std::string name = src_.substr(pos_, p - pos_);
                if (name != parent.name) fail("closing </" + name + "> inside <" + parent.name + ">");
                pos_ = p;
                skip_to(">");
                return;
            }
            // opening tag
            ++pos_;
            size_t p = pos_;
            while (p < src_.size() && src_[p] != '>' && src_[p] != '/' && !std::isspace((unsigned char)src_[p])) ++p;
            auto node = std::make_unique<XmlNode>();
            node->name = src_.substr(pos_, p - pos_);
            node->path = parent.path + "/" + node->name;
            if (node->name.empty()) fail("empty tag name");
            const size_t close = src_.find('>', p);
            if (close == std::string::npos) fail("unterminated tag <" + node->name);
            const bool self_closing = close > 0 && src_[close - 1] == '/';
            pos_ = close + 1;
            XmlNode* raw = node.get();
            parent.kids.push_back(std::move(node));
            if (!self_closing) parse_children(*raw);
        }
        if (!parent.name.empty()) fail("missing </" + parent.name + ">");
    }
};

}  // namespace clhost
