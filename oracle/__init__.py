"""Oracle package: CPU restatement of the reference path and drivers for the reference build.

Test infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU baseline)."""
