// Reader for the reference's input-deck format ([section] key = value, lists [a, b, c]) and
// the run description it produces. Used by salec_gpu_create_from_deck() so that a deck runs
// on the device without the reference's host code.
#pragma once
#include <map>
#include <string>
#include <vector>

namespace salec {

// Key/value store with the reference's parsing rules (src/io/InputParser.c:225-478):
//  - a line is trimmed; empty lines and lines starting with " # / - * are comments;
//  - "[name]" opens a section; keys without a '.' are prefixed with "section.";
//  - the key is the first run of characters that are neither '=' nor ' ';
//  - the value is the next run of characters that are none of # * " (and / in EOS files);
//  - trimming removes surrounding whitespace and also leading '.' characters;
//  - lookups are case-insensitive;
//  - list values "[a, b, c]": element k is the text between the k-th and (k+1)-th comma.
class Deck {
public:
    bool load(const std::string &path, bool eos_file, std::string &err);
    bool has(const std::string &key) const;
    std::string str(const std::string &key, const std::string &def) const;
    double num(const std::string &key, const std::string &def) const;
    int integer(const std::string &key, const std::string &def) const;
    double num_k(const std::string &key, int k, const std::string &def) const;
    int integer_k(const std::string &key, int k, const std::string &def) const;
    std::string str_k(const std::string &key, int k, const std::string &def) const;

private:
    std::map<std::string, std::string> kv_;
    const std::string *find(const std::string &key) const;
};

} // namespace salec
