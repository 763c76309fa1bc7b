// Host-only test driver: runs the lag kernel's table builder (build_lag_table) on launch
// descriptions read from stdin and prints each table, so that tests/test_lag_protocol.py can
// check the tables and replay the kernel's barrier protocol on the CPU. Calls no CUDA API.
//
// Input, one case per line: nreg J ntau npos, then reg[nreg], ent_acc[ntau], ent_w[ntau],
// pos[npos]. Output, one line per case: the table's ints, or "ERR <message>".
#include <iostream>
#include <string>
#include <vector>

#include "lag_host.hpp"

int main() {
    int nreg, J, ntau, npos;
    while (std::cin >> nreg >> J >> ntau >> npos) {
        std::vector<int> reg(64, -1), ent_acc(ntau), ent_w(ntau), pos(npos);
        for (int j = 0; j < nreg; j++) std::cin >> reg[j];
        for (int &v : ent_acc) std::cin >> v;
        for (int &v : ent_w) std::cin >> v;
        for (int &v : pos) std::cin >> v;
        std::vector<int> table;
        const std::string err = ddm::build_lag_table(nreg, reg.data(), ent_acc, ent_w, pos, J, &table);
        if (!err.empty()) {
            std::cout << "ERR " << err << "\n";
            continue;
        }
        for (size_t i = 0; i < table.size(); i++) std::cout << (i ? " " : "") << table[i];
        std::cout << "\n";
    }
    return 0;
}
