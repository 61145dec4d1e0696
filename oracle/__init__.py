"""TEST INFRASTRUCTURE: the CPU oracle of the flight-mode tick (a C++ restatement of the reference's scalar
algorithm, oracle/flight.cpp) and its numpy park (oracle/park.py). Only tests/, __graft_entry__.smoke() and bench.py's
CPU baseline use it, as the checker; the product (exact_ballpark_b200) never imports it."""
