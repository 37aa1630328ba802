#include "pd_deck.h"

#include <fstream>

namespace pdh {

namespace {
std::string trim(std::string line) {
    while (!line.empty() && line.back() == '\r') line.pop_back();
    line.erase(line.find_last_not_of(' ') + 1, std::string::npos);
    line.erase(0, line.find_first_not_of(' '));
    return line;
}
}  // namespace

bool DeckReader::Load(const std::string& path) {
    std::ifstream in(path.c_str());
    if (!in) return false;
    std::vector<std::string> raw;
    std::string line;
    while (std::getline(in, line)) raw.push_back(line);
    SetLines(raw);
    return true;
}

void DeckReader::SetLines(const std::vector<std::string>& raw) {
    lines_.clear();
    for (const std::string& l : raw) lines_.push_back(trim(l));
}

bool DeckReader::Find(const std::string& keyword) const {
    for (const std::string& l : lines_)
        if (l == keyword) return true;
    return false;
}

// pdDataManager::KeywordAppend, pdDataManager3.cpp:1553-1559
std::string keyword_append(const std::string& k, int i) {
    std::ostringstream o;
    o << i;
    return k + o.str();
}

}  // namespace pdh
