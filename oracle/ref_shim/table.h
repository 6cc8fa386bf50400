// Minimal stand-in for the contest's row-table helper, written for building the
// reference engine as a test oracle only. The engine mentions `Table` in one
// test-only helper (PlanImport::makeTable); the oracle never calls it.
#pragma once
#include <plan.h>
#include <stdexcept>
#include <vector>

struct Table {
    Table(std::vector<std::vector<Data>>, std::vector<DataType>) {}
    ColumnarTable to_columnar() const {
        throw std::runtime_error("table stub: row tables are not available in the oracle build");
    }
};
