// Stand-in for the part of Boost.PropertyTree the reference's deck loader uses
// (TEST INFRASTRUCTURE; Boost is not in this image).  Used by
// src/simulation_files/AMRSimulation.cpp:11-31 and AMRSimulation_load.cpp:3-258:
//   read_json(path, tree)                  throws json_parser_error
//   tree.get<T>(path)                      throws ptree_bad_path / ptree_bad_data
//   tree.get<T>(path, default)             default when absent or not convertible
//   tree.get_child(path)                   throws ptree_bad_path
//   child.get_value<T>()                   conversion of the node's own value
//   for (ptree::value_type& kv : tree)     children in file order (arrays: key "")
//   catch (ptree_error&)
// Values are kept as the text of the JSON token, as Boost's JSON reader does,
// and converted on access the way Boost's stream translator does: extraction
// from an istringstream must succeed and consume the whole text (trailing
// white space allowed); bool accepts 0/1 first, then true/false.
#ifndef FS_ORACLE_BOOST_PTREE_SHIM
#define FS_ORACLE_BOOST_PTREE_SHIM

#include <cctype>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace boost {
namespace property_tree {

struct ptree_error : public std::runtime_error {
    explicit ptree_error(const std::string& w) : std::runtime_error(w) {}
};
struct ptree_bad_path : public ptree_error {
    explicit ptree_bad_path(const std::string& w) : ptree_error("No such node (" + w + ")") {}
};
struct ptree_bad_data : public ptree_error {
    explicit ptree_bad_data(const std::string& w) : ptree_error("conversion of data failed (" + w + ")") {}
};
struct json_parser_error : public ptree_error {
    explicit json_parser_error(const std::string& w) : ptree_error(w) {}
};

namespace detail {

template <typename T>
inline bool convert(const std::string& s, T& out) {
    std::istringstream iss(s);
    iss >> out;
    if (!iss.eof()) iss >> std::ws;
    return !iss.fail() && !iss.bad() && iss.get() == std::char_traits<char>::eof();
}

template <>
inline bool convert<bool>(const std::string& s, bool& out) {
    {
        std::istringstream iss(s);
        iss >> out;
        if (!iss.fail()) {
            if (!iss.eof()) iss >> std::ws;
            if (!iss.fail() && iss.get() == std::char_traits<char>::eof()) return true;
        }
    }
    std::istringstream iss(s);
    iss.setf(std::ios_base::boolalpha);
    iss >> out;
    if (!iss.eof()) iss >> std::ws;
    return !iss.fail() && !iss.bad() && iss.get() == std::char_traits<char>::eof();
}

template <>
inline bool convert<std::string>(const std::string& s, std::string& out) {
    out = s;
    return true;
}

}  // namespace detail

class ptree {
public:
    typedef std::pair<const std::string, ptree> value_type;
    typedef std::vector<value_type>::iterator iterator;
    typedef std::vector<value_type>::const_iterator const_iterator;

    ptree() = default;

    iterator begin() { return children_.begin(); }
    iterator end() { return children_.end(); }
    const_iterator begin() const { return children_.begin(); }
    const_iterator end() const { return children_.end(); }

    const std::string& data() const { return data_; }
    void set_data(const std::string& d) { data_ = d; }
    ptree& push_back_child(const std::string& key, ptree&& child) {
        children_.emplace_back(key, std::move(child));
        return children_.back().second;
    }

    ptree& get_child(const std::string& path) {
        ptree* n = find(path);
        if (!n) throw ptree_bad_path(path);
        return *n;
    }
    const ptree& get_child(const std::string& path) const {
        const ptree* n = const_cast<ptree*>(this)->find(path);
        if (!n) throw ptree_bad_path(path);
        return *n;
    }

    template <typename T>
    T get_value() const {
        T v{};
        if (!detail::convert(data_, v)) throw ptree_bad_data(data_);
        return v;
    }

    template <typename T>
    T get(const std::string& path) const {
        return get_child(path).template get_value<T>();
    }

    template <typename T>
    T get(const std::string& path, const T& def) const {
        const ptree* n = const_cast<ptree*>(this)->find(path);
        if (!n) return def;
        T v{};
        if (!detail::convert(n->data_, v)) return def;
        return v;
    }

    std::string get(const std::string& path, const char* def) const {
        return get<std::string>(path, std::string(def));
    }

private:
    // '.'-separated path; the first child with each key
    ptree* find(const std::string& path) {
        ptree* cur = this;
        size_t pos = 0;
        while (cur) {
            size_t dot = path.find('.', pos);
            std::string key = path.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
            ptree* next = nullptr;
            for (auto& kv : cur->children_)
                if (kv.first == key) { next = &kv.second; break; }
            cur = next;
            if (dot == std::string::npos) break;
            pos = dot + 1;
        }
        return cur;
    }

    std::string data_;
    std::vector<value_type> children_;
};

namespace json_detail {

struct Reader {
    const std::string& s;
    size_t i = 0;
    explicit Reader(const std::string& text) : s(text) {}

    [[noreturn]] void fail(const char* what) {
        throw json_parser_error(std::string("json: ") + what + " at offset " + std::to_string(i));
    }
    void ws() {
        while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    }
    bool eat(char c) {
        ws();
        if (i < s.size() && s[i] == c) { ++i; return true; }
        return false;
    }
    std::string string_token() {
        if (!eat('"')) fail("expected string");
        std::string out;
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\') {
                if (i >= s.size()) fail("bad escape");
                char e = s[i++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (i + 4 > s.size()) fail("bad \\u escape");
                        unsigned v = std::stoul(s.substr(i, 4), nullptr, 16);
                        i += 4;
                        if (v < 0x80) out += char(v);
                        else if (v < 0x800) { out += char(0xC0 | (v >> 6)); out += char(0x80 | (v & 0x3F)); }
                        else { out += char(0xE0 | (v >> 12)); out += char(0x80 | ((v >> 6) & 0x3F)); out += char(0x80 | (v & 0x3F)); }
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (i >= s.size()) fail("unterminated string");
        ++i;
        return out;
    }
    void value(ptree& node) {
        ws();
        if (i >= s.size()) fail("unexpected end");
        char c = s[i];
        if (c == '{') {
            ++i;
            if (eat('}')) return;
            do {
                std::string key = string_token();
                if (!eat(':')) fail("expected ':'");
                ptree child;
                value(child);
                node.push_back_child(key, std::move(child));
            } while (eat(','));
            if (!eat('}')) fail("expected '}'");
        } else if (c == '[') {
            ++i;
            if (eat(']')) return;
            do {
                ptree child;
                value(child);
                node.push_back_child("", std::move(child));
            } while (eat(','));
            if (!eat(']')) fail("expected ']'");
        } else if (c == '"') {
            node.set_data(string_token());
        } else {
            // number, true, false, null: kept as their text
            size_t b = i;
            while (i < s.size() && !std::isspace(static_cast<unsigned char>(s[i])) && s[i] != ',' && s[i] != '}' &&
                   s[i] != ']')
                ++i;
            if (i == b) fail("expected value");
            node.set_data(s.substr(b, i - b));
        }
    }
};

}  // namespace json_detail

inline void read_json(const std::string& path, ptree& pt) {
    std::ifstream f(path);
    if (!f) throw json_parser_error("cannot open file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    json_detail::Reader r(text);
    ptree root;
    r.value(root);
    r.ws();
    if (r.i != text.size()) r.fail("trailing characters");
    pt = std::move(root);
}

}  // namespace property_tree
}  // namespace boost

#endif
