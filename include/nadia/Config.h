// Config.h -- drop-in for the reference's configuration-file reader
// (NADIA/include/Config.h, NADIA/src/Config.c++): "key = value" or
// "key value" lines, '#' starts a comment; typed getters set the status to
// FAILURE when a key is missing.
#ifndef NADIA_DROPIN_CONFIG_H
#define NADIA_DROPIN_CONFIG_H

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <list>
#include <map>
#include <sstream>
#include <string>

#include "types.h"

class Config {
public:
    typedef std::map<std::string, std::string> MapType; // the first line of a key wins

    explicit Config(std::string file_name)
    {
        std::ifstream file(file_name.c_str());
        if (!file.is_open()) {
            std::cout << "Could not open the file " << file_name << std::endl;
            status = FAILURE;
            return;
        }
        std::string line;
        while (std::getline(file, line)) {
            const size_t hash = line.find('#');
            if (hash != std::string::npos) line = line.substr(0, hash);
            size_t pos = line.find('=');
            if (pos == std::string::npos) pos = line.find(' ');
            if (pos == std::string::npos) continue;
            std::istringstream ks(line.substr(0, pos));
            std::string key;
            ks >> key;
            mapping.insert(std::make_pair(key, line.substr(pos + 1)));
        }
        status = SUCCESS;
    }

    int getStatus() { return status; }

    std::string getString(std::string key)
    {
        const std::string *v = find(key);
        if (!v) return "";
        std::istringstream s(*v);
        std::string value;
        s >> value;
        return value;
    }
    std::list<std::string> *getStringList(std::string key) { return tokens<std::string>(key); }
    std::list<int> *getIntList(std::string key) { return tokens<int>(key); }
    double getDouble(std::string key)
    {
        const std::string *v = find(key);
        return v ? std::atof(v->c_str()) : 0;
    }
    int getInt(std::string key)
    {
        const std::string *v = find(key);
        return v ? std::atoi(v->c_str()) : 0;
    }

private:
    MapType mapping;
    int status = FAILURE;

    const std::string *find(const std::string &key)
    {
        MapType::iterator it = mapping.find(key);
        if (it == mapping.end()) {
            std::cout << "Key:" << key << " not found in config file" << std::endl;
            status = FAILURE;
            return nullptr;
        }
        return &it->second;
    }

    template <class T>
    std::list<T> *tokens(const std::string &key)
    {
        const std::string *v = find(key);
        if (!v) return nullptr;
        std::list<T> *out = new std::list<T>;
        std::istringstream s(*v);
        std::string t;
        while (s >> t) out->push_back(convert<T>(t));
        if (out->empty()) {
            std::cout << "Key:" << key << " has no entries in the config file" << std::endl;
            status = FAILURE;
            delete out;
            return nullptr;
        }
        return out;
    }
    template <class T>
    static T convert(const std::string &t);
};

template <>
inline std::string Config::convert<std::string>(const std::string &t)
{
    return t;
}
template <>
inline int Config::convert<int>(const std::string &t)
{
    return std::atoi(t.c_str());
}

#endif
