// Headless stand-in for graphics/gui/header/residual_plot.h: records the
// monitored residuals of every check instead of plotting them.
#pragma once
#include <string>
#include <unordered_map>
#include <vector>

struct ConfigResidual;

class ResidualPlot {
public:
    struct Row {
        int iteration;
        double u, v, continuity, temperature, concentration;
    };
    std::vector<Row> rows;
    void resetState() { rows.clear(); }
    void clearPlot(int) {}
    void setName(const std::unordered_map<std::string, ConfigResidual>&) {}
    void add(int currentIteration, const std::unordered_map<std::string, ConfigResidual>& cfg);
};
