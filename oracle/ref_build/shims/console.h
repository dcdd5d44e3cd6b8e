// Headless stand-in for the reference GUI console (graphics/gui/header/console.h):
// same member names the solver calls, lines kept in memory for the driver.
#pragma once
#include <string>
#include <vector>

class Console {
public:
    std::vector<std::string> lines;
    float completionMs = 0.f;
    void addLine(const std::string& s) { lines.push_back(s); }
    void addCompletionMessage(const std::string& s) { lines.push_back(s); }
    void addCompletionTime(const std::string&, float& ms) { completionMs = ms; }
    void addSeparator() {}
    void clear() { lines.clear(); }
};
