"""CPU oracle for the HybriD-GM t_GPU path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
leg import this package, and only to check results against.  The product package
(simulador_quantico_b200) never imports it.

* circuit_lang   Python restatement of the reference's circuit language.
* cpu            ctypes bindings to the C restatement (oracle/sv_oracle.c)
                 and, when it was built here, to the reference's own engine
                 (oracle/_ref/libref_{f32,f64}.so).
* closed_forms   analytic states: H benchmark, Grover, QFT of a basis state.

The seeded benchmark circuits themselves are built by the product package's
simulador_quantico_b200/workloads.py (circuit strings only, no engine code).
"""
