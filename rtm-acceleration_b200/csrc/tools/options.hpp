// options.hpp -- the table of command-line options shared by the tools.
//
// Each entry binds one flag to the variable it sets.  Numeric and string
// entries may also raise a "given" flag, which the tools use for the
// velocity-header precedence rule (a value on the command line wins over the
// .hdr sidecar).  A terminal entry (--help, --list-engines) stops the scan and
// is returned to the caller, which acts on it before reading anything else.
#pragma once

#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace rtm_b200::cli {

class Options {
public:
    Options& text(const char* flag, std::string& dst, bool* given = nullptr) {
        return add(flag, true, false, [&dst, given](const std::string& v) { dst = v; mark(given); });
    }
    Options& integer(const char* flag, int& dst, bool* given = nullptr) {
        return add(flag, true, false, [&dst, given](const std::string& v) { dst = std::stoi(v); mark(given); });
    }
    Options& real(const char* flag, float& dst, bool* given = nullptr) {
        return add(flag, true, false, [&dst, given](const std::string& v) { dst = std::stof(v); mark(given); });
    }
    // A flag without a value that stores `value` into `dst`.
    Options& boolean(const char* flag, bool& dst, bool value = true) {
        return add(flag, false, false, [&dst, value](const std::string&) { dst = value; });
    }
    // A value mapped through a list of (word, code) pairs; other words are an error.
    Options& choice(const char* flag, int& dst, std::vector<std::pair<std::string, int>> words) {
        std::string f = flag;
        return add(flag, true, false, [&dst, f, words](const std::string& v) {
            std::string list;
            for (const auto& w : words) {
                if (w.first == v) { dst = w.second; return; }
                list += (list.empty() ? " " : "|") + w.first;
            }
            throw std::runtime_error(f + list);
        });
    }
    Options& terminal(const char* flag) {
        return add(flag, false, true, [](const std::string&) {});
    }

    // Applies argv[1..] in order.  Returns the terminal flag that stopped the
    // scan, or an empty string when every argument was consumed.
    std::string parse(int argc, char** argv) const {
        for (int i = 1; i < argc; ++i) {
            const std::string a = argv[i];
            const Entry* e = find(a);
            if (!e) throw std::runtime_error("unknown option: " + a);
            if (e->stop) return a;
            std::string v;
            if (e->takes_value) {
                if (i + 1 >= argc) throw std::runtime_error("missing value after " + a);
                v = argv[++i];
            }
            e->apply(v);
        }
        return {};
    }

private:
    struct Entry {
        std::string flag;
        bool takes_value;
        bool stop;
        std::function<void(const std::string&)> apply;
    };
    std::vector<Entry> table_;

    static void mark(bool* given) { if (given) *given = true; }
    Options& add(const char* flag, bool takes_value, bool stop, std::function<void(const std::string&)> f) {
        table_.push_back(Entry{flag, takes_value, stop, std::move(f)});
        return *this;
    }
    const Entry* find(const std::string& a) const {
        for (const auto& e : table_)
            if (e.flag == a) return &e;
        return nullptr;
    }
};

}  // namespace rtm_b200::cli
