// ReadConfig.hpp -- CConfig: the settings.cfg reader of the reference (include/ReadConfig.hpp:6-60)
// with the same key = value format: empty lines, lines starting with '#' and lines
// starting with '\r' are skipped, the first '=' splits key and value, and both are trimmed
// of surrounding blanks.  Unlike the reference, a missing file is reported by read()
// returning false (the reference prints and exits), so an embedding program decides.
#pragma once
#include <fstream>
#include <iostream>
#include <map>
#include <string>

class CConfig
{
public:
    std::string m_inputFileName;

    explicit CConfig(const std::string &str) : m_inputFileName(str) {}

    bool read(std::map<std::string, std::string> &option) const
    {
        std::ifstream input(m_inputFileName);
        if (!input.is_open()) {
            std::cerr << "Failed to open file " << m_inputFileName << std::endl;
            return false;
        }
        std::string line;
        while (std::getline(input, line)) {
            if (line.empty() || line[0] == '#' || line[0] == '\r') continue;
            const size_t eq = line.find('=');
            if (eq == std::string::npos) {
                std::cerr << "Invalid line: " << line << std::endl;
                continue;
            }
            option[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
        }
        return true;
    }

    static std::string trim(const std::string &s)
    {
        const char *blank = " \t\r\n\f\v";
        const size_t a = s.find_first_not_of(blank);
        if (a == std::string::npos) return std::string();
        const size_t b = s.find_last_not_of(blank);
        return s.substr(a, b - a + 1);
    }
};
