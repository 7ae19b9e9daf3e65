// Header-only stand-in for the subset of libconfig++ that the reference
// (src/GeneralModel/antelope.cpp, SBEs.h, Materials/*.h) uses, so the
// unmodified reference sources compile without libconfig installed.
// Test infrastructure only: on the include path of the oracle/_ref build.
//
// Grammar handled (libconfig text format): settings `name = value` or
// `name : value` with optional `;`/`,` terminators; groups `{}`, lists `()`,
// arrays `[]` of scalars; booleans (true/false, any case); integers (decimal,
// 0x hex, optional L suffix); floats (a '.' or an exponent); strings with C
// escapes and adjacent-literal concatenation; comments `#`, `//`, `/* */`.
//
// Type rules follow libconfig without auto-conversion: reading an integer
// setting as double (or a float as int) throws SettingTypeException, and
// lookupValue() returns false on a missing name or a type mismatch.
//
// The reference redefines the token `complex` as a macro around this header
// (SBEs.h:17-23), so the token is not used anywhere below.
#ifndef ORACLE_REFSHIM_LIBCONFIG_HPP
#define ORACLE_REFSHIM_LIBCONFIG_HPP

#include <cctype>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace libconfig {

class ConfigException : public std::exception {
public:
    const char *what() const noexcept override { return "ConfigException"; }
};

class Setting;

class SettingException : public ConfigException {
public:
    explicit SettingException(const std::string &path) : path_(path) {}
    const char *getPath() const { return path_.c_str(); }
    const char *what() const noexcept override { return "SettingException"; }

private:
    std::string path_;
};

class SettingNotFoundException : public SettingException {
public:
    explicit SettingNotFoundException(const std::string &path) : SettingException(path) {}
    const char *what() const noexcept override { return "SettingNotFoundException"; }
};

class SettingTypeException : public SettingException {
public:
    explicit SettingTypeException(const std::string &path) : SettingException(path) {}
    const char *what() const noexcept override { return "SettingTypeException"; }
};

class FileIOException : public ConfigException {
public:
    const char *what() const noexcept override { return "FileIOException"; }
};

class ParseException : public ConfigException {
public:
    ParseException(const std::string &file, int line, const std::string &err)
        : file_(file), line_(line), err_(err) {}
    const char *getFile() const { return file_.c_str(); }
    int getLine() const { return line_; }
    const char *getError() const { return err_.c_str(); }
    const char *what() const noexcept override { return "ParseException"; }

private:
    std::string file_;
    int line_;
    std::string err_;
};

class Setting {
public:
    enum Type { TypeNone, TypeInt, TypeInt64, TypeFloat, TypeString, TypeBoolean,
                TypeGroup, TypeArray, TypeList };

    Type getType() const { return type_; }
    const char *getName() const { return name_.c_str(); }
    int getLength() const
    {
        return (type_ == TypeGroup || type_ == TypeArray || type_ == TypeList)
                   ? static_cast<int>(children_.size()) : 0;
    }
    bool isGroup() const { return type_ == TypeGroup; }
    bool isArray() const { return type_ == TypeArray; }
    bool isList() const { return type_ == TypeList; }
    bool isAggregate() const { return isGroup() || isArray() || isList(); }
    bool isNumber() const { return type_ == TypeInt || type_ == TypeInt64 || type_ == TypeFloat; }

    Setting &operator[](int idx) const
    {
        if (!isAggregate() || idx < 0 || idx >= static_cast<int>(children_.size()))
            throw SettingNotFoundException(path_ + "[" + std::to_string(idx) + "]");
        return *children_[idx];
    }
    Setting &operator[](const char *name) const
    {
        Setting *s = find(name);
        if (!s) throw SettingNotFoundException(path_ + "." + name);
        return *s;
    }
    Setting &operator[](const std::string &name) const { return (*this)[name.c_str()]; }

    bool exists(const char *name) const { return find(name) != nullptr; }
    bool exists(const std::string &name) const { return exists(name.c_str()); }

    Setting &lookup(const char *path) const
    {
        const Setting *cur = this;
        std::string p(path);
        size_t pos = 0;
        while (pos <= p.size()) {
            size_t dot = p.find('.', pos);
            std::string part = p.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
            cur = &(*cur)[part.c_str()];
            if (dot == std::string::npos) break;
            pos = dot + 1;
        }
        return const_cast<Setting &>(*cur);
    }
    Setting &lookup(const std::string &path) const { return lookup(path.c_str()); }

    operator bool() const { need(TypeBoolean); return bval_; }
    operator int() const { needInt(); return static_cast<int>(ival_); }
    operator unsigned int() const { needInt(); return static_cast<unsigned int>(ival_); }
    operator long() const { needInt(); return static_cast<long>(ival_); }
    operator long long() const { needInt(); return ival_; }
    operator double() const { need(TypeFloat); return fval_; }
    operator float() const { need(TypeFloat); return static_cast<float>(fval_); }
    operator std::string() const { need(TypeString); return sval_; }
    const char *c_str() const { need(TypeString); return sval_.c_str(); }

    template <typename T>
    bool lookupValue(const char *name, T &value) const
    {
        Setting *s = find(name);
        if (!s) return false;
        try {
            value = s->template as<T>();
        } catch (const SettingTypeException &) {
            return false;
        }
        return true;
    }
    template <typename T>
    bool lookupValue(const std::string &name, T &value) const { return lookupValue(name.c_str(), value); }

    // construction (used by the parser below)
    Setting() = default;
    Type type_ = TypeNone;
    std::string name_, path_;
    bool bval_ = false;
    long long ival_ = 0;
    double fval_ = 0.0;
    std::string sval_;
    std::vector<std::unique_ptr<Setting>> children_;

private:
    template <typename T> T as() const { return static_cast<T>(*this); }

    Setting *find(const char *name) const
    {
        if (type_ != TypeGroup) return nullptr;
        for (const auto &c : children_)
            if (c->name_ == name) return c.get();
        return nullptr;
    }
    void need(Type t) const
    {
        if (type_ != t) throw SettingTypeException(path_);
    }
    void needInt() const
    {
        if (type_ != TypeInt && type_ != TypeInt64) throw SettingTypeException(path_);
    }
};

template <> inline std::string Setting::as<std::string>() const { return static_cast<std::string>(*this); }

namespace refshim_detail {

class Parser {
public:
    Parser(const std::string &text, const std::string &file) : s_(text), file_(file) {}

    void parseSettings(Setting &group, char close)
    {
        for (;;) {
            skip();
            if (pos_ >= s_.size()) {
                if (close) fail("unexpected end of file");
                return;
            }
            if (close && s_[pos_] == close) { ++pos_; return; }
            std::string name = parseName();
            skip();
            if (pos_ < s_.size() && (s_[pos_] == '=' || s_[pos_] == ':')) ++pos_;
            else fail("expected '=' or ':' after setting name");
            auto child = std::unique_ptr<Setting>(new Setting());
            child->name_ = name;
            child->path_ = group.path_.empty() ? name : group.path_ + "." + name;
            parseValue(*child);
            for (const auto &c : group.children_)
                if (c->name_ == name) fail("duplicate setting name '" + name + "'");
            group.children_.push_back(std::move(child));
            skip();
            if (pos_ < s_.size() && (s_[pos_] == ';' || s_[pos_] == ',')) ++pos_;
        }
    }

private:
    const std::string &s_;
    std::string file_;
    size_t pos_ = 0;

    int line() const
    {
        int l = 1;
        for (size_t i = 0; i < pos_ && i < s_.size(); ++i) l += (s_[i] == '\n');
        return l;
    }
    [[noreturn]] void fail(const std::string &msg) const { throw ParseException(file_, line(), msg); }

    void skip()
    {
        while (pos_ < s_.size()) {
            char c = s_[pos_];
            if (c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\f' || c == '\v') { ++pos_; continue; }
            if (c == '#' || (c == '/' && pos_ + 1 < s_.size() && s_[pos_ + 1] == '/')) {
                while (pos_ < s_.size() && s_[pos_] != '\n') ++pos_;
                continue;
            }
            if (c == '/' && pos_ + 1 < s_.size() && s_[pos_ + 1] == '*') {
                size_t e = s_.find("*/", pos_ + 2);
                if (e == std::string::npos) fail("unterminated comment");
                pos_ = e + 2;
                continue;
            }
            break;
        }
    }

    std::string parseName()
    {
        size_t b = pos_;
        if (pos_ < s_.size() && (std::isalpha(static_cast<unsigned char>(s_[pos_])) || s_[pos_] == '*')) ++pos_;
        else fail("expected a setting name");
        while (pos_ < s_.size()) {
            char c = s_[pos_];
            if (std::isalnum(static_cast<unsigned char>(c)) || c == '_' || c == '-' || c == '*') ++pos_;
            else break;
        }
        return s_.substr(b, pos_ - b);
    }

    void parseValue(Setting &out)
    {
        skip();
        if (pos_ >= s_.size()) fail("expected a value");
        char c = s_[pos_];
        if (c == '{') {
            ++pos_;
            out.type_ = Setting::TypeGroup;
            parseSettings(out, '}');
        } else if (c == '(' || c == '[') {
            char close = (c == '(') ? ')' : ']';
            out.type_ = (c == '(') ? Setting::TypeList : Setting::TypeArray;
            ++pos_;
            int idx = 0;
            for (;;) {
                skip();
                if (pos_ < s_.size() && s_[pos_] == close) { ++pos_; break; }
                auto child = std::unique_ptr<Setting>(new Setting());
                child->path_ = out.path_ + "[" + std::to_string(idx++) + "]";
                parseValue(*child);
                if (out.type_ == Setting::TypeArray) {
                    if (child->isAggregate()) fail("arrays hold scalars only");
                    if (!out.children_.empty() && out.children_[0]->type_ != child->type_)
                        fail("array elements must share one type");
                }
                out.children_.push_back(std::move(child));
                skip();
                if (pos_ < s_.size() && s_[pos_] == ',') { ++pos_; continue; }
                if (pos_ < s_.size() && s_[pos_] == close) { ++pos_; break; }
                fail("expected ',' or closing bracket");
            }
        } else if (c == '"') {
            out.type_ = Setting::TypeString;
            out.sval_.clear();
            while (pos_ < s_.size() && s_[pos_] == '"') {
                ++pos_;
                while (pos_ < s_.size() && s_[pos_] != '"') {
                    char d = s_[pos_++];
                    if (d == '\\' && pos_ < s_.size()) {
                        char e = s_[pos_++];
                        switch (e) {
                            case 'n': d = '\n'; break;
                            case 't': d = '\t'; break;
                            case 'r': d = '\r'; break;
                            case 'f': d = '\f'; break;
                            default: d = e; break;
                        }
                    }
                    out.sval_.push_back(d);
                }
                if (pos_ >= s_.size()) fail("unterminated string");
                ++pos_;
                skip();
            }
        } else {
            size_t b = pos_;
            while (pos_ < s_.size()) {
                char d = s_[pos_];
                if (std::isalnum(static_cast<unsigned char>(d)) || d == '.' || d == '+' || d == '-' || d == '_') ++pos_;
                else break;
            }
            std::string tok = s_.substr(b, pos_ - b);
            if (tok.empty()) fail("unexpected character");
            std::string low;
            for (char d : tok) low.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(d))));
            if (low == "true" || low == "false") {
                out.type_ = Setting::TypeBoolean;
                out.bval_ = (low == "true");
                return;
            }
            bool hex = low.size() > 2 && (low.compare(0, 2, "0x") == 0 || low.compare(0, 3, "-0x") == 0);
            bool isfloat = !hex && (low.find('.') != std::string::npos || low.find('e') != std::string::npos);
            char *end = nullptr;
            if (isfloat) {
                out.type_ = Setting::TypeFloat;
                out.fval_ = std::strtod(tok.c_str(), &end);
            } else {
                std::string t = tok;
                bool i64 = false;
                if (!t.empty() && (t.back() == 'L' || t.back() == 'l')) {
                    i64 = true;
                    t.pop_back();
                    if (!t.empty() && (t.back() == 'L' || t.back() == 'l')) t.pop_back();
                }
                out.type_ = i64 ? Setting::TypeInt64 : Setting::TypeInt;
                out.ival_ = std::strtoll(t.c_str(), &end, 0);
                if (end && *end == '\0') return;
                fail("malformed number '" + tok + "'");
            }
            if (!end || *end != '\0') fail("malformed value '" + tok + "'");
        }
    }
};

}  // namespace refshim_detail

class Config {
public:
    Config() { root_.type_ = Setting::TypeGroup; }
    void readFile(const char *filename)
    {
        std::ifstream in(filename);
        if (!in) throw FileIOException();
        std::stringstream buf;
        buf << in.rdbuf();
        std::string text = buf.str();
        Setting fresh;
        fresh.type_ = Setting::TypeGroup;
        refshim_detail::Parser p(text, filename);
        p.parseSettings(fresh, 0);
        root_.children_ = std::move(fresh.children_);
    }
    void readFile(const std::string &filename) { readFile(filename.c_str()); }
    Setting &getRoot() const { return const_cast<Setting &>(root_); }
    bool exists(const char *path) const
    {
        try {
            root_.lookup(path);
            return true;
        } catch (const SettingNotFoundException &) {
            return false;
        }
    }
    bool exists(const std::string &path) const { return exists(path.c_str()); }
    Setting &lookup(const char *path) const { return root_.lookup(path); }
    Setting &lookup(const std::string &path) const { return root_.lookup(path.c_str()); }
    template <typename T>
    bool lookupValue(const char *path, T &value) const
    {
        try {
            value = static_cast<T>(root_.lookup(path));
        } catch (const SettingException &) {
            return false;
        }
        return true;
    }
    template <typename T>
    bool lookupValue(const std::string &path, T &value) const { return lookupValue(path.c_str(), value); }

private:
    Setting root_;
};

}  // namespace libconfig

#endif
