// Keyword deck reader with the semantics of pdDataManager::FindKeyword and
// pdDataManager::ReadKeyword (pdDataManager.h:270-421): a keyword line is
// matched after trimming spaces at both ends, its values are read from the
// next line with operator>> in order, and the first occurrence decides.
// Unlike the reference, a trailing carriage return is stripped too, so decks
// with CR/LF line ends read the same as LF decks, and failures are returned
// as status codes.
#pragma once

#include <sstream>
#include <string>
#include <vector>

namespace pdh {

class DeckReader {
public:
    // reads the whole file; false if it cannot be opened
    bool Load(const std::string& path);
    void SetLines(const std::vector<std::string>& raw);
    bool Find(const std::string& keyword) const;
    // 0 ok, 1 keyword missing, 2 value missing at the position
    template <typename T>
    int Read(const std::string& keyword, int position, T& value) const {
        for (size_t k = 0; k < lines_.size(); ++k) {
            if (lines_[k] != keyword) continue;
            std::istringstream iss(k + 1 < lines_.size() ? lines_[k + 1] : std::string());
            for (int i = 1; !iss.eof(); ++i) {
                iss >> value;
                if (i < position && iss.eof()) return 2;
                if (i == position) return 0;
            }
            return 2;
        }
        return 1;
    }
    const std::vector<std::string>& Lines() const { return lines_; }

private:
    std::vector<std::string> lines_;
};

std::string keyword_append(const std::string& k, int i);

}  // namespace pdh
