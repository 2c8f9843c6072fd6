"""TEST ORACLE ONLY.

CPU restatement of the reference's hot-path algorithms (cs_oracle.c) and
bridges to the reference's own code compiled from its sources (_ref/).  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
package, always as the checker; the product (cellshard_b200) never does.
"""
