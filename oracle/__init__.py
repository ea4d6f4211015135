"""Test oracle package (CPU restatement of the reference path). Test infrastructure only."""
